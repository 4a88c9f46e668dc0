// pz_capi.cu -- C ABI entry points (include/palzilla_b200.h) over the kernels.
#include <cstdio>
#include <cstring>
#include <string>

#include "pz_bvh.cuh"
#include "pz_capi_internal.h"
#include "pz_sort.cuh"

namespace pz {
namespace {
thread_local std::string g_last_error;
}  // namespace

int fail(int code, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

int cuda_fail(cudaError_t e, const char* where)
{
    return fail(PZ_ERR_CUDA, "%s: %s (%s)", where, cudaGetErrorString(e), cudaGetErrorName(e));
}

void clear_error() { g_last_error.clear(); }
}  // namespace pz

using namespace pz;

extern "C" int pz_version(void) { return 1; }

extern "C" const char* pz_last_error(void) { return g_last_error.c_str(); }

extern "C" int pz_scratch_status(const void* scratch_dev, uint32_t* status_out, pz_stream_t stream)
{
    if (!scratch_dev || !status_out) return fail(PZ_ERR_INVALID_ARGUMENT, "pz_scratch_status: null pointer");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(e, "pz_scratch_status: stream synchronize");
    e = cudaMemcpy(status_out, scratch_dev, sizeof(uint32_t), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "pz_scratch_status: copy");
    clear_error();
    return PZ_OK;
}

// ---------------------------------------------------------------- sort
extern "C" size_t pz_onesweep_scratch_bytes(uint32_t n) { return sort::scratch_bytes(n); }

extern "C" int pz_onesweep_sort(void* keys_dev, uint32_t* values_dev, void* tmp_keys_dev, uint32_t* tmp_values_dev,
                                uint32_t n, int key_bytes, int start_bit, int end_bit, void* scratch_dev,
                                size_t scratch_bytes, pz_stream_t stream)
{
    if (key_bytes != 4 && key_bytes != 8)
        return fail(PZ_ERR_INVALID_ARGUMENT, "pz_onesweep_sort: key_bytes must be 4 or 8 (got %d)", key_bytes);
    if (start_bit < 0 || end_bit <= start_bit || end_bit > 8 * key_bytes)
        return fail(PZ_ERR_INVALID_ARGUMENT, "pz_onesweep_sort: bad bit range [%d, %d)", start_bit, end_bit);
    const int nPasses = sort::num_passes(start_bit, end_bit);
    if (start_bit + 8 * nPasses > 8 * key_bytes + 7 || nPasses > sort::kMaxPasses)
        return fail(PZ_ERR_INVALID_ARGUMENT, "pz_onesweep_sort: too many digit passes");
    if (n == 0) { clear_error(); return PZ_OK; }
    if (!keys_dev || !tmp_keys_dev || !scratch_dev || (values_dev && !tmp_values_dev))
        return fail(PZ_ERR_INVALID_ARGUMENT, "pz_onesweep_sort: null buffer");
    if (scratch_bytes < sort::scratch_bytes(n))
        return fail(PZ_ERR_SCRATCH_TOO_SMALL, "pz_onesweep_sort: scratch %zu < required %zu", scratch_bytes,
                    sort::scratch_bytes(n));
    auto misaligned = [](const void* p, size_t a) { return (reinterpret_cast<uintptr_t>(p) % a) != 0; };
    if (misaligned(keys_dev, key_bytes) || misaligned(tmp_keys_dev, key_bytes) || misaligned(values_dev, 4) ||
        misaligned(tmp_values_dev, 4) || misaligned(scratch_dev, 16))
        return fail(PZ_ERR_INVALID_ARGUMENT, "pz_onesweep_sort: misaligned buffer");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    auto* h = static_cast<sort::Header*>(scratch_dev);
    auto* lb = reinterpret_cast<unsigned long long*>(static_cast<char*>(scratch_dev) + sort::kHeaderBytes);
    cudaError_t e = cudaMemsetAsync(h, 0, sizeof(sort::Header), s);
    if (e == cudaSuccess) {
        if (key_bytes == 8) {
            auto* k = static_cast<unsigned long long*>(keys_dev);
            e = sort::launch_hist<unsigned long long>(k, n, start_bit, nPasses, h, lb, s);
            if (e == cudaSuccess)
                e = sort::launch_passes<unsigned long long>(k, values_dev, static_cast<unsigned long long*>(tmp_keys_dev),
                                                            tmp_values_dev, n, start_bit, nPasses, h, lb, s);
        } else {
            auto* k = static_cast<uint32_t*>(keys_dev);
            e = sort::launch_hist<uint32_t>(k, n, start_bit, nPasses, h, lb, s);
            if (e == cudaSuccess)
                e = sort::launch_passes<uint32_t>(k, values_dev, static_cast<uint32_t*>(tmp_keys_dev), tmp_values_dev,
                                                  n, start_bit, nPasses, h, lb, s);
        }
    }
    if (e != cudaSuccess) return cuda_fail(e, "pz_onesweep_sort");
    clear_error();
    return PZ_OK;
}

// ---------------------------------------------------------------- LBVH
extern "C" size_t pz_bvh_scratch_bytes(int n) { return n < 0 ? 0 : bvh::scratch_bytes((uint32_t)n); }

extern "C" int pz_bvh_build(const pz_triangle* triangles_dev, int n, uint32_t build_option,
                            pz_internal_node* internals_dev, uint32_t* root_dev, void* scratch_dev,
                            size_t scratch_bytes, pz_stream_t stream)
{
    if (n < 0) return fail(PZ_ERR_INVALID_ARGUMENT, "pz_bvh_build: negative triangle count");
    if (!root_dev || !scratch_dev || (n > 0 && !triangles_dev) || (n > 1 && !internals_dev))
        return fail(PZ_ERR_INVALID_ARGUMENT, "pz_bvh_build: null buffer");
    if (scratch_bytes < bvh::scratch_bytes((uint32_t)n))
        return fail(PZ_ERR_SCRATCH_TOO_SMALL, "pz_bvh_build: scratch %zu < required %zu", scratch_bytes,
                    bvh::scratch_bytes((uint32_t)n));
    if ((reinterpret_cast<uintptr_t>(triangles_dev) & 3) || (reinterpret_cast<uintptr_t>(internals_dev) & 15) ||
        (reinterpret_cast<uintptr_t>(root_dev) & 3) || (reinterpret_cast<uintptr_t>(scratch_dev) & 255))
        return fail(PZ_ERR_INVALID_ARGUMENT, "pz_bvh_build: misaligned buffer (internals need 16-byte, scratch 256-byte alignment)");
    cudaError_t e = bvh::build(reinterpret_cast<const Tri*>(triangles_dev), (uint32_t)n, build_option,
                               reinterpret_cast<Node*>(internals_dev), root_dev, scratch_dev,
                               reinterpret_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_fail(e, "pz_bvh_build");
    clear_error();
    return PZ_OK;
}

extern "C" int pz_bvh_debug_views(void* scratch_dev, int n, const uint64_t** sorted_dev, const uint8_t** deltas_dev,
                                  pz_aabb* aabb_out, pz_stream_t stream)
{
    if (!scratch_dev || n < 0) return fail(PZ_ERR_INVALID_ARGUMENT, "pz_bvh_debug_views: bad argument");
    bvh::Layout L = bvh::layout(scratch_dev, (uint32_t)n);
    if (sorted_dev) *sorted_dev = reinterpret_cast<const uint64_t*>(L.keys);
    if (deltas_dev) *deltas_dev = L.deltas;
    if (aabb_out) {
        cudaError_t e = cudaStreamSynchronize(reinterpret_cast<cudaStream_t>(stream));
        uint32_t enc[6];
        if (e == cudaSuccess) e = cudaMemcpy(enc, L.s->aabb_enc, sizeof(enc), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return cuda_fail(e, "pz_bvh_debug_views");
        auto unord = [](uint32_t u) {
            uint32_t b = (u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u;
            float f;
            memcpy(&f, &b, 4);
            return f;
        };
        aabb_out->lower = pz_float3{unord(~enc[0]), unord(~enc[1]), unord(~enc[2])};
        aabb_out->upper = pz_float3{unord(enc[3]), unord(enc[4]), unord(enc[5])};
    }
    clear_error();
    return PZ_OK;
}
