// pz_sort_static.cu -- pz_onesweep_sort_static: the onesweep sort on a static device
// scratch array, for callers that cannot allocate device memory at call time.
//
// The scratch (sort header + look-back rows for PZ_ONESWEEP_STATIC_MAX_KEYS keys) is a
// __device__ array of this library.  A __device__ symbol has one address per CUDA context
// (the module is loaded into each context separately), so every call looks the address up
// with cudaGetSymbolAddress in the context current on the calling thread: a host that makes
// its own contexts, or re-creates the primary context after cudaDeviceReset, gets the
// address that belongs to the context it is running in.  The look-up allocates nothing; the
// first one in a context may load this library's module into it.  The sort itself is
// pz_onesweep_sort, unchanged, given that array as its scratch.  Nothing in the array has to
// start at zero: every call clears the header with cudaMemsetAsync on its stream and the
// histogram kernel clears the look-back rows it uses.  The array is shared by every call in
// a context, so calls whose work overlaps on the GPU (different streams without ordering)
// race on it.
#include "pz_capi_internal.h"
#include "pz_sort.cuh"

namespace pz {
namespace {

constexpr uint32_t kStaticMaxKeys = PZ_ONESWEEP_STATIC_MAX_KEYS;
constexpr size_t kStaticLookback = (size_t)((kStaticMaxKeys + sort::kTile - 1) / sort::kTile) * sort::kRadix * 8;
constexpr size_t kStaticBytes = sort::kHeaderBytes + ((kStaticLookback + 255) & ~(size_t)255);

__device__ __align__(256) unsigned char g_sort_scratch[kStaticBytes];

// Device address of g_sort_scratch in the current context.
int static_scratch(void** out)
{
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_sort_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "pz_onesweep_sort_static: cudaGetSymbolAddress");
    if (!p) return fail(PZ_ERR_CUDA, "pz_onesweep_sort_static: null scratch symbol address");
    *out = p;
    return PZ_OK;
}

}  // namespace
}  // namespace pz

using namespace pz;

static_assert(kStaticBytes >= sort::kHeaderBytes + 256, "static scratch");

extern "C" int pz_onesweep_sort_static(void* keys_dev, uint32_t* values_dev, void* tmp_keys_dev,
                                       uint32_t* tmp_values_dev, uint32_t n, int key_bytes, int start_bit,
                                       int end_bit, uint32_t* status_dev, pz_stream_t stream)
{
    if (n > kStaticMaxKeys)
        return fail(PZ_ERR_SCRATCH_TOO_SMALL,
                    "pz_onesweep_sort_static: n = %u exceeds the static scratch capacity of %u keys "
                    "(use pz_onesweep_sort with caller-owned scratch)",
                    n, kStaticMaxKeys);
    if (status_dev && (reinterpret_cast<uintptr_t>(status_dev) & 3))
        return fail(PZ_ERR_INVALID_ARGUMENT, "pz_onesweep_sort_static: misaligned status word");
    void* scratch = nullptr;
    int r = static_scratch(&scratch);
    if (r != PZ_OK) return r;
    if (sort::scratch_bytes(n) > kStaticBytes)
        return fail(PZ_ERR_SCRATCH_TOO_SMALL, "pz_onesweep_sort_static: scratch %zu < required %zu", kStaticBytes,
                    sort::scratch_bytes(n));
    r = pz_onesweep_sort(keys_dev, values_dev, tmp_keys_dev, tmp_values_dev, n, key_bytes, start_bit, end_bit, scratch,
                         kStaticBytes, stream);
    if (r != PZ_OK || !status_dev) return r;
    // the sort's status word (look-back spin limit) is the first word of the header
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    cudaError_t e = n == 0 ? cudaMemsetAsync(status_dev, 0, sizeof(uint32_t), s)
                           : cudaMemcpyAsync(status_dev, scratch, sizeof(uint32_t), cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) return cuda_fail(e, "pz_onesweep_sort_static: status copy");
    clear_error();
    return PZ_OK;
}
