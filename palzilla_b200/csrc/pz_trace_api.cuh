// pz_trace_api.cuh -- batch ray query launchers (see pz_trace.cu).
#pragma once
#include "pz_common.cuh"

namespace pz {
cudaError_t launch_trace_closest(const Node* nodes, const uint32_t* root, const Tri* tris, uint32_t n, const float* ro,
                                 const float* rd, float* t, float* uv, uint32_t* tri, float* ng, uint32_t* status,
                                 cudaStream_t s);
cudaError_t launch_trace_any(const Node* nodes, const uint32_t* root, const Tri* tris, uint32_t n, const float* ro,
                             const float* rd, const float* tmax, uint8_t* hit, cudaStream_t s);
}  // namespace pz
