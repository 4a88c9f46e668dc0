// ref_gpu_lbvh.cu -- TEST INFRASTRUCTURE ONLY.
//
// The reference's own LBVH kernels (minimum_lbvh.cu: getSceneAABB, buildMortons,
// computeDeltas, build), compiled for sm_100a from the reference sources where they lie by
// oracle/build_ref_gpu.sh, with host entry points that launch them as
// BVHGPUBuilder::build does (minimum_lbvh.h:798-886) through the CUDA runtime instead of
// Orochi.  The sort between the Morton keys and the deltas is left to the caller (the
// reference's onesweep reorder takes its tile index from blockIdx.x and spins without bound
// on its predecessors, tinyhiponesweep.h:341-381, which is safe only under in-order block
// dispatch; it is not run here).  Included by oracle/ref_gpu_main.cu, which is the one
// translation unit the recipe compiles.  Used by tests/ and bench.py's reference-kernel
// workload.
#include <cuda_runtime.h>

#include "minimum_lbvh.cu"

namespace {
inline unsigned blocks256(long long n) { return (unsigned)((n + 255) / 256); }
}  // namespace

// scene AABB (minimum_lbvh.h:818-829): the empty box, then getSceneAABB.
extern "C" int pzg_scene_aabb(AABB* aabb_dev, const Triangle* tris_dev, int n, cudaStream_t s)
{
    // AABB::empty() (minimum_lbvh.h:225-236) is device-only in a CUDA build: the same six floats
    static const float empty[6] = {MINIMUM_LBVH_FLT_MAX, MINIMUM_LBVH_FLT_MAX, MINIMUM_LBVH_FLT_MAX,
                                   -MINIMUM_LBVH_FLT_MAX, -MINIMUM_LBVH_FLT_MAX, -MINIMUM_LBVH_FLT_MAX};
    static_assert(sizeof(AABB) == sizeof(empty), "AABB layout");
    cudaError_t e = cudaMemcpyAsync(aabb_dev, empty, sizeof(AABB), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return (int)e;
    if (n > 0) getSceneAABB<<<blocks256(n), 256, 0, s>>>(aabb_dev, tris_dev, n);
    return (int)cudaGetLastError();
}

// Morton keys (minimum_lbvh.h:831-844).
extern "C" int pzg_build_mortons(IndexedMorton* out_dev, const Triangle* tris_dev, int n, const AABB* aabb_dev,
                                 uint32_t build_option, cudaStream_t s)
{
    if (n > 0) buildMortons<<<blocks256(n), 256, 0, s>>>(out_dev, tris_dev, n, aabb_dev, build_option);
    return (int)cudaGetLastError();
}

// Deltas of the sorted keys, the 0xFF fill of the nodes, and the bottom-up build
// (minimum_lbvh.h:850-879).
extern "C" int pzg_deltas_and_build(NodeIndex* root_dev, InternalNode* internals_dev, uint8_t* deltas_dev,
                                    const Triangle* tris_dev, int n, const IndexedMorton* sorted_dev, cudaStream_t s)
{
    if (n < 2) return (int)cudaErrorInvalidValue;
    computeDeltas<<<blocks256(n - 1), 256, 0, s>>>(deltas_dev, sorted_dev, n);
    cudaError_t e = cudaMemsetAsync(internals_dev, 0xFF, sizeof(InternalNode) * (size_t)(n - 1), s);
    if (e != cudaSuccess) return (int)e;
    build<<<blocks256(n - 1), 256, 0, s>>>(root_dev, internals_dev, tris_dev, n, deltas_dev, sorted_dev);
    return (int)cudaGetLastError();
}
