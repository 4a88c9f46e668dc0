// ref_gpu_main.cu -- TEST INFRASTRUCTURE ONLY.
//
// The reference's own frame kernels (main_gpu.cu: photonTrace, lookupFlatten,
// reorderSpecularPath, solveSpecularPath_K1..4, pack), compiled for sm_100a from the
// reference sources where they lie by oracle/build_ref_gpu.sh, with host entry points that
// launch them as PKRenderer::step does (pk.h:1436-1570) through the CUDA runtime instead of
// Orochi's Shader::launch.  Kernel parameters that are structs of the reference (PathCache,
// EventDescriptor, CauchyDispersion) are passed as the byte images the kernels expect, as
// Orochi passes them.  Built twice: with the compiler's default FMA contraction (the
// reference's run-time compile, used for timing) and with -fmad=false (its CPU float
// arithmetic, used for parity).  Used by tests/ and bench.py's reference-kernel workload.
#include <cuda_runtime.h>

// One translation unit for all the reference's kernels: its headers define non-inline
// functions (minimum_lbvh.h:42-43), which two units would define twice.
#include "ref_gpu_lbvh.cu"

// The reference calls the pre-Volta warp vote __any (pk.h:1151), which sm_70+ spells with a mask.
#define __any(p) __any_sync(0xFFFFFFFFu, (p))

#include "main_gpu.cu"

namespace {

// PathCache in a CUDA build (pk.h:227-402): the cell step, then three TypedBuffer
// {T* data; size_t size : 63, isDevice : 1} (typedbuffer.h:19-24).
struct PathCacheImage {
    float step;
    uint32_t pad;
    void* hashes;
    uint64_t hashesSize;
    void* paths;
    uint64_t pathsSize;
    void* count;
    uint64_t countSize;
};
static_assert(sizeof(PathCacheImage) == sizeof(PathCache), "PathCache layout");
static_assert(sizeof(PathCache::TrianglePath) == 56, "TrianglePath layout");
static_assert(sizeof(EventDescriptor) == 4 && sizeof(CauchyDispersion) == 8, "argument layouts");

PathCacheImage cache_image(void* hashes, void* paths, void* count, float step)
{
    const uint64_t dev = 1ull << 63;
    return PathCacheImage{step, 0u, hashes, PathCache::CACHE_STORAGE_COUNT | dev, paths,
                          PathCache::CACHE_STORAGE_COUNT | dev, count, 1ull | dev};
}

inline unsigned div_up(uint64_t n, uint64_t d) { return (unsigned)((n + d - 1) / d); }

}  // namespace

extern "C" int pzg_path_cache_capacity(void) { return (int)PathCache::CACHE_STORAGE_COUNT; }
extern "C" int pzg_triangle_path_bytes(void) { return (int)sizeof(PathCache::TrianglePath); }
extern "C" size_t pzg_stack_buffer_bytes(void)
{
    return sizeof(NodeIndex) * (size_t)STACK_BUFFER_MAX_WARPS * 32 * STACK_BUFFER_MAX_ELEMENT;
}

// photonTrace (main_gpu.cu:56-211): one 256-thread block per triangle (pk.h:1440-1458).
// hashes_dev (u32 x 2^22) and count_dev are cleared by the caller (PathCache::clear);
// stack_dev is pzg_stack_buffer_bytes() of zeros (StackBufferAllocator, pk.h:1119-1126).
extern "C" int pzg_photon_trace(const NodeIndex* root_dev, const InternalNode* internals_dev, const Triangle* tris_dev,
                                const TriangleAttrib* attribs_dev, int n_tris, const float* p_light3, float eta_min,
                                float eta_max, int iteration, void* hashes_dev, void* paths_dev, void* count_dev,
                                float step, float min_throughput, NodeIndex* stack_dev, cudaStream_t s)
{
    float3 pl = make_float3(p_light3[0], p_light3[1], p_light3[2]);
    PathCacheImage pc = cache_image(hashes_dev, paths_dev, count_dev, step);
    float3* debugPoints = nullptr;
    int* debugCount = nullptr;
    void* args[] = {&root_dev, &internals_dev, &tris_dev, &attribs_dev, &pl, &eta_min, &eta_max, &iteration,
                    &pc,       &min_throughput, &debugPoints, &debugCount, &stack_dev};
    return (int)cudaLaunchKernel((const void*)photonTrace, dim3(n_tris), dim3(PHOTON_BLOCK_SIZE), args, 0, s);
}

// lookupFlatten (main_gpu.cu:373-416), 16 x 16 blocks over the image (pk.h:1490-1500).
extern "C" int pzg_lookup_flatten(uint32_t events, SpecularPath* paths_dev, IndexedSpecularPath* indexed_dev,
                                  uint32_t* counter_dev, const FirstDiffuse* fds_dev, int width, int height,
                                  void* hashes_dev, void* paths_cache_dev, void* count_dev, float step, cudaStream_t s)
{
    int2 size = make_int2(width, height);
    PathCacheImage pc = cache_image(hashes_dev, paths_cache_dev, count_dev, step);
    void* args[] = {&events, &paths_dev, &indexed_dev, &counter_dev, &fds_dev, &size, &pc};
    return (int)cudaLaunchKernel((const void*)lookupFlatten, dim3(div_up(width, 16), div_up(height, 16)), dim3(16, 16),
                                 args, 0, s);
}

// reorderSpecularPath (main_gpu.cu:515-525).
extern "C" int pzg_reorder(IndexedSpecularPath* indexed_dev, SpecularPath* dst_dev, const SpecularPath* src_dev, int n,
                           cudaStream_t s)
{
    if (n <= 0) return 0;
    reorderSpecularPath<<<div_up(n, 256), 256, 0, s>>>(indexed_dev, dst_dev, src_dev, n);
    return (int)cudaGetLastError();
}

// solveSpecularPath_K<K> (main_gpu.cu:418-497), one thread per work item (pk.h:1548-1566).
extern "C" int pzg_solve_specular(int K, float4* accum_dev, SpecularPath* paths_dev, uint32_t n,
                                  const FirstDiffuse* fds_dev, const NodeIndex* root_dev,
                                  const InternalNode* internals_dev, const Triangle* tris_dev,
                                  const TriangleAttrib* attribs_dev, const float* p_light3, float light_intensity,
                                  float radiance_clamp, void* hashes_dev, void* paths_cache_dev, void* count_dev,
                                  float step, uint32_t events, float cauchy_a, float cauchy_b, int iteration,
                                  cudaStream_t s)
{
    if (n == 0) return 0;
    float3 pl = make_float3(p_light3[0], p_light3[1], p_light3[2]);
    PathCacheImage pc = cache_image(hashes_dev, paths_cache_dev, count_dev, step);
    const float cauchy[2] = {cauchy_a, cauchy_b};  // CauchyDispersion {m_A, m_B} (pk.h:935-949)
    void* args[] = {&accum_dev, &paths_dev, &n,  &fds_dev, &root_dev, &internals_dev, &tris_dev,  &attribs_dev,
                    &pl,        &light_intensity, &radiance_clamp, &pc, &events, (void*)cauchy, &iteration};
    const void* fn = nullptr;
    switch (K) {
        case 1: fn = (const void*)solveSpecularPath_K1; break;
        case 2: fn = (const void*)solveSpecularPath_K2; break;
        case 3: fn = (const void*)solveSpecularPath_K3; break;
        case 4: fn = (const void*)solveSpecularPath_K4; break;
        default: return (int)cudaErrorInvalidValue;
    }
    return (int)cudaLaunchKernel(fn, dim3(div_up(n, 256)), dim3(256), args, 0, s);
}

// pack (main_gpu.cu:499-513).
extern "C" int pzg_pack(uint32_t* pixels_dev, float4* accum_dev, int n, cudaStream_t s)
{
    if (n <= 0) return 0;
    pack<<<div_up(n, 256), 256, 0, s>>>(pixels_dev, accum_dev, n);
    return (int)cudaGetLastError();
}
