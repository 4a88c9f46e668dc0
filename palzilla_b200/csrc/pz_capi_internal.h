// pz_capi_internal.h -- error helpers shared by the C ABI translation units.
#pragma once
#include <cuda_runtime.h>
#include <cstdarg>

#include "../../include/palzilla_b200.h"

namespace pz {
int fail(int code, const char* fmt, ...);
int cuda_fail(cudaError_t e, const char* where);
void clear_error();
}  // namespace pz
