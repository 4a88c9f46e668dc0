// pz_bvh.cu -- LBVH construction (minimum_lbvh.h:798-886 / minimum_lbvh.cu).
//
// Pipeline, all on the caller's stream, no host synchronisation:
//   memset(header)                  zero the sort header (histograms, counters, status, AABB)
//   k_scene_aabb                    getSceneAABB (minimum_lbvh.cu:38-66)
//   k_morton_hist                   buildMortons (minimum_lbvh.cu:68-92) fused with the
//                                   radix-sort histogram and the look-back clear
//   4 x k_pass                      onesweep sort of u64 {morton, index} on bits [0, 32)
//   k_deltas                        computeDeltas (minimum_lbvh.cu:94-102) + handshake init
//   k_build                         build_lbvh (minimum_lbvh.h:293-370), one thread per leaf
//
// The output InternalNode array and root are bit-exact with the reference builder
// run on the stable sort order.  Differences from the reference's kernels:
//  * the scene AABB is accumulated as order-preserving integers, so a zeroed header
//    is the empty box and no initialising copy is needed;
//  * triangles are staged through shared memory with 16-byte loads;
//  * the second-arrival handshake uses a separate u32 array, so the node array needs
//    no 0xFF memset (every field of every node is written by the build);
//  * the build launches ceil(n / 256) blocks over all n leaves (the reference launches
//    ceil((n - 1) / 256) and so skips leaf n - 1 when n % 256 == 1).
#include "pz_bvh.cuh"
#include "pz_sort.cuh"

namespace pz {
namespace bvh {

// order-preserving float <-> u32
PZ_D uint32_t ord(float f)
{
    uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
PZ_D float unord(uint32_t u) { return __uint_as_float((u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u); }

PZ_D Box load_scene_box(const Scratch* s)
{
    const uint32_t* e = s->aabb_enc;
    Box b;
    b.lo = mk3(unord(~e[0]), unord(~e[1]), unord(~e[2]));
    b.hi = mk3(unord(e[3]), unord(e[4]), unord(e[5]));
    return b;
}

// Stage 256 triangles (9216 B) of this block through shared memory with 16-byte loads.
PZ_D void stage_tris(float* sm, const Tri* tris, uint32_t first, uint32_t count)
{
    const float* src = reinterpret_cast<const float*>(tris) + (size_t)first * 9;
    const uint32_t nf = count * 9;
    // 16-byte path when the source is aligned; otherwise scalar loads.
    if ((reinterpret_cast<uintptr_t>(src) & 15) == 0) {
        const uint32_t nv = nf / 4;
        for (uint32_t i = threadIdx.x; i < nv; i += blockDim.x)
            reinterpret_cast<float4*>(sm)[i] = __ldg(reinterpret_cast<const float4*>(src) + i);
        for (uint32_t i = nv * 4 + threadIdx.x; i < nf; i += blockDim.x) sm[i] = __ldg(src + i);
    } else {
        for (uint32_t i = threadIdx.x; i < nf; i += blockDim.x) sm[i] = __ldg(src + i);
    }
}

constexpr int kBlock = 256;

__global__ void __launch_bounds__(kBlock) k_scene_aabb(const Tri* __restrict__ tris, uint32_t n, Scratch* s)
{
    __shared__ __align__(16) float sm[kBlock * 9];
    Box b = box_empty();
    for (uint32_t first = blockIdx.x * kBlock; first < n; first += gridDim.x * kBlock) {
        uint32_t cnt = min((uint32_t)kBlock, n - first);
        __syncthreads();
        stage_tris(sm, tris, first, cnt);
        __syncthreads();
        if (threadIdx.x < cnt) {
            const float* t = sm + threadIdx.x * 9;
            box_extend(b, mk3(t[0], t[1], t[2]));
            box_extend(b, mk3(t[3], t[4], t[5]));
            box_extend(b, mk3(t[6], t[7], t[8]));
        }
    }
    float v[6] = {b.lo.x, b.lo.y, b.lo.z, b.hi.x, b.hi.y, b.hi.z};
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int c = 0; c < 3; c++) v[c] = fminf(v[c], __shfl_xor_sync(0xFFFFFFFFu, v[c], o));
#pragma unroll
        for (int c = 3; c < 6; c++) v[c] = fmaxf(v[c], __shfl_xor_sync(0xFFFFFFFFu, v[c], o));
    }
    if ((threadIdx.x & 31) == 0 && v[0] <= v[3]) {
        for (int c = 0; c < 3; c++) atomicMax(&s->aabb_enc[c], ~ord(v[c]));
        for (int c = 3; c < 6; c++) atomicMax(&s->aabb_enc[c], ord(v[c]));
    }
}

// splat3 / encodeMortonCode, minimum_lbvh.h:173-195, 249-254
PZ_D unsigned long long splat3(uint32_t a)
{
    unsigned long long x = a & 0x1fffff;
    x = (x | x << 32) & 0x1f00000000ffffull;
    x = (x | x << 16) & 0x1f0000ff0000ffull;
    x = (x | x << 8) & 0x100f00f00f00f00full;
    x = (x | x << 4) & 0x10c30c30c30c30c3ull;
    x = (x | x << 2) & 0x1249249249249249ull;
    return x;
}
PZ_D unsigned long long encode_morton(const Box& b, float3 p)
{
    float3 q = ((p - b.lo) / (b.hi - b.lo)) * 2097152.0f;
    // float -> int conversion truncates and saturates (NaN -> 0), then clamps
    int cx = max(0, min(__float2int_rz(q.x), 0x1FFFFF));
    int cy = max(0, min(__float2int_rz(q.y), 0x1FFFFF));
    int cz = max(0, min(__float2int_rz(q.z), 0x1FFFFF));
    return splat3((uint32_t)cx) | splat3((uint32_t)cy) << 1 | splat3((uint32_t)cz) << 2;
}

__global__ void __launch_bounds__(kBlock) k_morton_hist(const Tri* __restrict__ tris, uint32_t n, uint32_t opt,
                                                        Scratch* s, unsigned long long* __restrict__ keys,
                                                        unsigned long long* lookback, size_t lookbackWords)
{
    __shared__ __align__(16) float sm[kBlock * 9];
    __shared__ uint32_t hist[4 * sort::kRadix];
    for (int i = threadIdx.x; i < 4 * sort::kRadix; i += kBlock) hist[i] = 0;
    sort::clear_lookback(lookback, lookbackWords);
    const Box scene = load_scene_box(s);
    const Box unit{mk3(-1.f, -1.f, -1.f), mk3(1.f, 1.f, 1.f)};
    for (uint32_t first = blockIdx.x * kBlock; first < n; first += gridDim.x * kBlock) {
        uint32_t cnt = min((uint32_t)kBlock, n - first);
        __syncthreads();
        stage_tris(sm, tris, first, cnt);
        __syncthreads();
        if (threadIdx.x < cnt) {
            const float* t = sm + threadIdx.x * 9;
            float3 v0 = mk3(t[0], t[1], t[2]), v1 = mk3(t[3], t[4], t[5]), v2 = mk3(t[6], t[7], t[8]);
            float3 center = (v0 + v1 + v2) / 3.0f;
            uint32_t key;
            if (opt & PZ_BUILD_OPTION_USE_NORMAL) {  // GPU packing, minimum_lbvh.cu:79-86
                float3 ng = normalize(cross(v1 - v0, v2 - v0));
                uint32_t nM = (uint32_t)(encode_morton(unit, ng) >> 31);
                uint32_t pM = (uint32_t)(encode_morton(scene, center) >> 31);
                key = (nM & 0xFFFFFFC0u) | (pM >> 26);
            } else {
                key = (uint32_t)(encode_morton(scene, center) >> 31);  // upper 32 of 63 bits
            }
            uint32_t idx = first + threadIdx.x;
            keys[idx] = (unsigned long long)key | ((unsigned long long)idx << 32);
#pragma unroll
            for (int p = 0; p < 4; p++) atomicAdd(&hist[p * sort::kRadix + ((key >> (8 * p)) & 0xFFu)], 1u);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 4 * sort::kRadix; i += kBlock) {
        uint32_t c = hist[i];
        if (c) atomicAdd(&s->sort.hist[0][0] + i, c);
    }
}

__global__ void __launch_bounds__(kBlock) k_deltas(const unsigned long long* __restrict__ sorted, uint32_t n,
                                                   uint8_t* __restrict__ deltas, uint32_t* __restrict__ flags)
{
    uint32_t i = blockIdx.x * kBlock + threadIdx.x;
    if (i + 1 >= n) return;
    uint32_t a = (uint32_t)sorted[i], b = (uint32_t)sorted[i + 1];
    deltas[i] = (uint8_t)(32 - __clz(a ^ b));  // delta, minimum_lbvh.h:140-143 (__clz(0) == 32)
    flags[i] = 0xFFFFFFFFu;
}

__global__ void __launch_bounds__(kBlock) k_build(Node* __restrict__ nodes, uint32_t* __restrict__ rootOut,
                                                  const Tri* __restrict__ tris, uint32_t n,
                                                  const uint8_t* __restrict__ deltas, uint32_t* flags,
                                                  const unsigned long long* __restrict__ sorted)
{
    const uint32_t i_leaf = blockIdx.x * kBlock + threadIdx.x;
    if (n == 0) {
        if (i_leaf == 0) *rootOut = kInvalidNode;
        return;
    }
    if (i_leaf >= n) return;
    const uint32_t nInternals = n - 1;
    const uint32_t triIndex = (uint32_t)(sorted[i_leaf] >> 32);
    uint32_t lower = i_leaf, upper = i_leaf;
    uint32_t node = make_node(triIndex, true);
    const float* t = reinterpret_cast<const float*>(tris) + (size_t)triIndex * 9;
    Box box = box_empty();
    box_extend(box, mk3(__ldg(t + 0), __ldg(t + 1), __ldg(t + 2)));
    box_extend(box, mk3(__ldg(t + 3), __ldg(t + 4), __ldg(t + 5)));
    box_extend(box, mk3(__ldg(t + 6), __ldg(t + 7), __ldg(t + 8)));
    bool isRoot = true;
    while (upper - lower < nInternals) {
        uint32_t dL = 0 < lower ? __ldg(deltas + lower - 1) : 0xFFFFFFFFu;
        uint32_t dR = upper < nInternals ? __ldg(deltas + upper) : 0xFFFFFFFFu;
        int goLeft = dL < dR ? 1 : 0;
        uint32_t parent = goLeft ? (lower - 1) : upper;
        Node* P = nodes + parent;
        P->children[goLeft] = node;
        P->boxes[goLeft] = box;
        if (!is_leaf(node)) nodes[node_idx(node)].parent = make_node(parent, false);
        uint32_t other = goLeft ? upper : lower;
        __threadfence();
        other = atomicExch(flags + parent, other);
        if (other == 0xFFFFFFFFu) { isRoot = false; break; }
        __threadfence();
        lower = min(lower, other);
        upper = max(upper, other);
        P->context = upper < nInternals ? upper : 0xFFFFFFFFu;
        node = make_node(parent, false);
        // the sibling half was written by another thread: read it from L2
        const float* ob = reinterpret_cast<const float*>(&P->boxes[goLeft ^ 1]);
        Box o;
        o.lo = mk3(__ldcg(ob + 0), __ldcg(ob + 1), __ldcg(ob + 2));
        o.hi = mk3(__ldcg(ob + 3), __ldcg(ob + 4), __ldcg(ob + 5));
        box_extend(box, o);
    }
    if (isRoot) {
        *rootOut = node;
        if (nInternals > 0) nodes[node_idx(node)].parent = kInvalidNode;
    }
}

size_t scratch_bytes(uint32_t n)
{
    size_t b = sizeof(Scratch);
    b = (b + 255) & ~(size_t)255;
    b += (sort::lookback_bytes(n) + 255) & ~(size_t)255;
    b += 2 * (((size_t)n * 8 + 255) & ~(size_t)255);  // keys + tmp
    b += ((size_t)n + 255) & ~(size_t)255;            // deltas
    b += ((size_t)n * 4 + 255) & ~(size_t)255;        // flags
    return b;
}

Layout layout(void* scratch, uint32_t n)
{
    Layout L;
    char* p = static_cast<char*>(scratch);
    L.s = reinterpret_cast<Scratch*>(p);
    p += (sizeof(Scratch) + 255) & ~(size_t)255;
    L.lookback = reinterpret_cast<unsigned long long*>(p);
    p += (sort::lookback_bytes(n) + 255) & ~(size_t)255;
    L.keys = reinterpret_cast<unsigned long long*>(p);
    p += ((size_t)n * 8 + 255) & ~(size_t)255;
    L.tmp = reinterpret_cast<unsigned long long*>(p);
    p += ((size_t)n * 8 + 255) & ~(size_t)255;
    L.deltas = reinterpret_cast<uint8_t*>(p);
    p += ((size_t)n + 255) & ~(size_t)255;
    L.flags = reinterpret_cast<uint32_t*>(p);
    return L;
}

cudaError_t build(const Tri* tris, uint32_t n, uint32_t opt, Node* nodes, uint32_t* root, void* scratch,
                  cudaStream_t st, Stage stopAfter)
{
    Layout L = layout(scratch, n);
    cudaError_t e = cudaMemsetAsync(L.s, 0, sizeof(Scratch), st);
    if (e != cudaSuccess) return e;
    if (n == 0) {
        k_build<<<1, kBlock, 0, st>>>(nodes, root, tris, 0, nullptr, nullptr, nullptr);
        return cudaGetLastError();
    }
    const int grid = (int)min((uint32_t)(kNumSMs * 8), (n + kBlock - 1) / kBlock);
    k_scene_aabb<<<grid, kBlock, 0, st>>>(tris, n, L.s);
    k_morton_hist<<<grid, kBlock, 0, st>>>(tris, n, opt, L.s, L.keys, L.lookback, (size_t)sort::num_tiles(n) * sort::kRadix);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (stopAfter == Stage::kKeys) return cudaSuccess;
    e = sort::launch_passes<unsigned long long>(L.keys, nullptr, L.tmp, nullptr, n, 0, 4, &L.s->sort, L.lookback, st);
    if (e != cudaSuccess) return e;
    if (stopAfter == Stage::kSorted) return cudaSuccess;
    const int g = (int)((n + kBlock - 1) / kBlock);
    k_deltas<<<g, kBlock, 0, st>>>(L.keys, n, L.deltas, L.flags);
    k_build<<<g, kBlock, 0, st>>>(nodes, root, tris, n, L.deltas, L.flags, L.keys);
    return cudaGetLastError();
}

}  // namespace bvh
}  // namespace pz
