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
#include <cuda/atomic>

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

// Streams the vertex array as 16-byte loads: 12 floats (4 vertices) per step, whose
// axis pattern is fixed (x y z x | y z x y | z x y z).
__global__ void __launch_bounds__(kBlock) k_scene_aabb(const Tri* __restrict__ tris, uint32_t n, Scratch* s)
{
    const float* f = reinterpret_cast<const float*>(tris);
    const uint64_t nf = (uint64_t)n * 9;
    float lo[3] = {kFltMax, kFltMax, kFltMax}, hi[3] = {-kFltMax, -kFltMax, -kFltMax};
    auto ext = [&](int a, float v) {
        lo[a] = fminf(lo[a], v);
        hi[a] = fmaxf(hi[a], v);
    };
    const bool aligned = (reinterpret_cast<uintptr_t>(f) & 15) == 0;
    const uint64_t groups = aligned ? nf / 12 : 0;
    const float4* q = reinterpret_cast<const float4*>(f);
    const uint64_t stride = (uint64_t)gridDim.x * kBlock;
    uint64_t g = (uint64_t)blockIdx.x * kBlock + threadIdx.x;
    for (; g + stride < groups; g += 2 * stride) {
        const float4 a0 = __ldcs(q + 3 * g), b0 = __ldcs(q + 3 * g + 1), c0 = __ldcs(q + 3 * g + 2);
        const uint64_t h = g + stride;
        const float4 a1 = __ldcs(q + 3 * h), b1 = __ldcs(q + 3 * h + 1), c1 = __ldcs(q + 3 * h + 2);
        ext(0, a0.x); ext(1, a0.y); ext(2, a0.z); ext(0, a0.w); ext(1, b0.x); ext(2, b0.y);
        ext(0, b0.z); ext(1, b0.w); ext(2, c0.x); ext(0, c0.y); ext(1, c0.z); ext(2, c0.w);
        ext(0, a1.x); ext(1, a1.y); ext(2, a1.z); ext(0, a1.w); ext(1, b1.x); ext(2, b1.y);
        ext(0, b1.z); ext(1, b1.w); ext(2, c1.x); ext(0, c1.y); ext(1, c1.z); ext(2, c1.w);
    }
    for (; g < groups; g += stride) {
        const float4 a0 = __ldcs(q + 3 * g), b0 = __ldcs(q + 3 * g + 1), c0 = __ldcs(q + 3 * g + 2);
        ext(0, a0.x); ext(1, a0.y); ext(2, a0.z); ext(0, a0.w); ext(1, b0.x); ext(2, b0.y);
        ext(0, b0.z); ext(1, b0.w); ext(2, c0.x); ext(0, c0.y); ext(1, c0.z); ext(2, c0.w);
    }
    for (uint64_t i = groups * 12 + (uint64_t)blockIdx.x * kBlock + threadIdx.x; i < nf; i += stride)
        ext((int)(i % 3), __ldg(f + i));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int c = 0; c < 3; c++) {
            lo[c] = fminf(lo[c], __shfl_xor_sync(0xFFFFFFFFu, lo[c], o));
            hi[c] = fmaxf(hi[c], __shfl_xor_sync(0xFFFFFFFFu, hi[c], o));
        }
    }
    __shared__ float red[kBlock / 32][6];
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0)
        for (int c = 0; c < 3; c++) { red[w][c] = lo[c]; red[w][3 + c] = hi[c]; }
    __syncthreads();
    if (threadIdx.x < 6) {
        const int c = threadIdx.x;
        float v = red[0][c];
        for (int k = 1; k < kBlock / 32; k++) v = c < 3 ? fminf(v, red[k][c]) : fmaxf(v, red[k][c]);
        // blocks without data contribute +-FLT_MAX, which never wins
        atomicMax(&s->aabb_enc[c], c < 3 ? ~ord(v) : ord(v));
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

// Writes a finished node with four 16-byte stores (whole 32-byte sectors).
PZ_D void store_node(Node* dst, const uint32_t c[2], const Box b[2], uint32_t parent, uint32_t context)
{
    float4* q = reinterpret_cast<float4*>(dst);
    q[0] = make_float4(__uint_as_float(c[0]), __uint_as_float(c[1]), b[0].lo.x, b[0].lo.y);
    q[1] = make_float4(b[0].lo.z, b[0].hi.x, b[0].hi.y, b[0].hi.z);
    q[2] = make_float4(b[1].lo.x, b[1].lo.y, b[1].lo.z, b[1].hi.x);
    q[3] = make_float4(b[1].hi.y, b[1].hi.z, __uint_as_float(parent), __uint_as_float(context));
}

// One thread per leaf climbs while it is the second to arrive at a node.  Each arriver
// leaves its child index and box in its side's 32-byte slot of the parent's pending record
// (a whole DRAM sector: no partial writes into the node array); the exchange on the
// handshake word is acquire-release, so the second arriver sees the first one's slot.  A finished node is kept in
// registers until its own parent is known and then written whole, once.
__global__ void __launch_bounds__(kBlock) k_build(Node* __restrict__ nodes, uint32_t* __restrict__ rootOut,
                                                  const Tri* __restrict__ tris, uint32_t n,
                                                  const uint8_t* __restrict__ deltas, uint32_t* flags,
                                                  const unsigned long long* __restrict__ sorted,
                                                  float4* __restrict__ pendingRecs)
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
    bool pending = false;  // `node` is internal, finished, and not yet written
    uint32_t pc[2], pctx = 0;
    Box pb[2];
    bool isRoot = true;
    // A node whose children are both leaves (leaf i climbs right, leaf i + 1 climbs left: a
    // local maximum of the deltas, about a third of the nodes of random keys) is made by
    // leaf i's thread alone, with the box of leaf i + 1 from its triangle; leaf i + 1's
    // thread stops.  The node is the one the handshake would make (same children, boxes,
    // parent and escape link), without its pending slots and flag exchange.
    if (nInternals > 0) {
        const auto goes_left = [&](uint32_t l) {
            const uint32_t a = 0 < l ? __ldg(deltas + l - 1) : 0xFFFFFFFFu;
            const uint32_t b = l < nInternals ? __ldg(deltas + l) : 0xFFFFFFFFu;
            return a < b;
        };
        const bool left = goes_left(i_leaf);
        if (!left && goes_left(i_leaf + 1)) {
            const uint32_t tri1 = (uint32_t)(sorted[i_leaf + 1] >> 32);
            const float* t1 = reinterpret_cast<const float*>(tris) + (size_t)tri1 * 9;
            Box b1 = box_empty();
            box_extend(b1, mk3(__ldg(t1 + 0), __ldg(t1 + 1), __ldg(t1 + 2)));
            box_extend(b1, mk3(__ldg(t1 + 3), __ldg(t1 + 4), __ldg(t1 + 5)));
            box_extend(b1, mk3(__ldg(t1 + 6), __ldg(t1 + 7), __ldg(t1 + 8)));
            pc[0] = node;
            pc[1] = make_node(tri1, true);
            pb[0] = box;
            pb[1] = b1;
            upper = i_leaf + 1;
            pctx = upper < nInternals ? upper : 0xFFFFFFFFu;
            pending = true;
            node = make_node(i_leaf, false);
            box_extend(box, b1);
        } else if (left && i_leaf > 0 && !goes_left(i_leaf - 1)) {
            return;  // leaf i - 1's thread makes the parent
        }
    }
    while (upper - lower < nInternals) {
        const uint32_t dL = 0 < lower ? __ldg(deltas + lower - 1) : 0xFFFFFFFFu;
        const uint32_t dR = upper < nInternals ? __ldg(deltas + upper) : 0xFFFFFFFFu;
        const int goLeft = dL < dR ? 1 : 0;
        const uint32_t parent = goLeft ? (lower - 1) : upper;
        if (pending) store_node(nodes + node_idx(node), pc, pb, make_node(parent, false), pctx);
        pending = false;
        float4* mine = pendingRecs + 4 * (size_t)parent + 2 * goLeft;  // this side's slot
        __stcg(mine + 0, make_float4(box.lo.x, box.lo.y, box.lo.z, box.hi.x));
        __stcg(mine + 1, make_float4(box.hi.y, box.hi.z, __uint_as_float(node), 0.0f));
        cuda::atomic_ref<uint32_t, cuda::thread_scope_device> hs(flags[parent]);
        const uint32_t other = hs.exchange(goLeft ? upper : lower, cuda::memory_order_acq_rel);
        if (other == 0xFFFFFFFFu) { isRoot = false; break; }
        lower = min(lower, other);
        upper = max(upper, other);
        const float4* theirs = pendingRecs + 4 * (size_t)parent + 2 * (goLeft ^ 1);
        const float4 r0 = __ldcg(theirs + 0), r1 = __ldcg(theirs + 1);
        Box o;
        o.lo = mk3(r0.x, r0.y, r0.z);
        o.hi = mk3(r0.w, r1.x, r1.y);
        // children and boxes by side, with selects (constant indices keep them in registers)
        const uint32_t theirChild = __float_as_uint(r1.z);
        pc[0] = goLeft ? theirChild : node;
        pc[1] = goLeft ? node : theirChild;
        pb[0] = goLeft ? o : box;
        pb[1] = goLeft ? box : o;
        pctx = upper < nInternals ? upper : 0xFFFFFFFFu;
        pending = true;
        node = make_node(parent, false);
        box_extend(box, o);
    }
    if (isRoot) {
        *rootOut = node;
        if (pending) store_node(nodes + node_idx(node), pc, pb, kInvalidNode, pctx);
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
    b += ((size_t)n * 64 + 255) & ~(size_t)255;       // pending records (two 32-byte slots)
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
    p += ((size_t)n * 4 + 255) & ~(size_t)255;
    L.pending = reinterpret_cast<float4*>(p);
    return L;
}

cudaError_t build(const Tri* tris, uint32_t n, uint32_t opt, Node* nodes, uint32_t* root, void* scratch,
                  cudaStream_t st, Stage stopAfter)
{
    Layout L = layout(scratch, n);
    cudaError_t e = cudaMemsetAsync(L.s, 0, sizeof(Scratch), st);
    if (e != cudaSuccess) return e;
    if (n == 0) {
        k_build<<<1, kBlock, 0, st>>>(nodes, root, tris, 0, nullptr, nullptr, nullptr, nullptr);
        return cudaGetLastError();
    }
    const int grid = (int)min((uint32_t)(num_sms() * 8), (n + kBlock - 1) / kBlock);
    k_scene_aabb<<<num_sms() * 8, kBlock, 0, st>>>(tris, n, L.s);
    k_morton_hist<<<grid, kBlock, 0, st>>>(tris, n, opt, L.s, L.keys, L.lookback, (size_t)sort::num_tiles(n) * sort::kRadix);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (stopAfter == Stage::kKeys) return cudaSuccess;
    e = sort::launch_passes<unsigned long long>(L.keys, nullptr, L.tmp, nullptr, n, 0, 4, &L.s->sort, L.lookback, st);
    if (e != cudaSuccess) return e;
    if (stopAfter == Stage::kSorted) return cudaSuccess;
    const int g = (int)((n + kBlock - 1) / kBlock);
    k_deltas<<<g, kBlock, 0, st>>>(L.keys, n, L.deltas, L.flags);
    k_build<<<g, kBlock, 0, st>>>(nodes, root, tris, n, L.deltas, L.flags, L.keys, L.pending);
    return cudaGetLastError();
}

}  // namespace bvh
}  // namespace pz
