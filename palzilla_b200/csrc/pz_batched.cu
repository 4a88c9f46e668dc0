// pz_batched.cu -- batched persistent specular solver (binned wavelengths).
//
// Same work items and results as the plain solver (one (pixel, tuple) work item solved
// for every wavelength bin with solveSpecularPath<K> semantics, pk.h / main_gpu.cu:418-497),
// organised for the GPU in three launches:
//  * k_probe, one thread per (item, probe bin): the plain path's solve from the photon's
//    barycentrics at the centre, first and last bin;
//  * k_phase1, one thread per item: the branch of roots through the centre bin (the probe's
//    root, or an unconstrained Newton solve from the photon's barycentrics), its
//    derivative in eta from the same Jacobian (implicit-function theorem), the two end-bin
//    roots refined from the tangent prediction, and a quadratic prediction of every bin's
//    root.  Bins whose predicted root lies outside a triangle by more than the prediction
//    error (plus the bin next to each edge crossing) need no solve; an item with no bin
//    left is skipped.  Items whose branch disagrees with a probe (the plain path reaches
//    another root there, or rejects where the branch is deep inside), whose solves did not
//    converge, whose prediction is strongly nonlinear, or whose Jacobian is near a fold,
//    take the plain per-bin solve for every bin.  Items with work are appended to a record
//    list with warp-aggregated atomics;
//  * phase 2, in waves of three kernels (see the phase-2 section): k_p2_solve, one warp per
//    record, lanes over the record's bins to solve in rank order: bins deep inside the
//    triangles refine the predicted root, every other bin runs the plain path's solve from
//    the photon's barycentrics, so its accept / reject decision is the plain one; then
//    admissibility, with optional FP64 polish of roots whose relative Jacobian determinant is
//    below a threshold; k_p2_vis, one warp per round of accepted roots of one record:
//    visibility shared by the warp (one BVH query per path segment with the segment fattened
//    to cover every root's segment; each root tests only those candidates); k_p2_contrib, one
//    thread per visible root: dAdw and the spectral accumulation.
// The unit is compiled without FMA contraction: with the reference's operation order in
// every Newton step, the image equals the reference's float arithmetic up to the order
// of the float atomics.
#include "pz_batched.cuh"
#include "pz_batched_api.cuh"

namespace pz {
namespace batched {

// Compile-time choices measured by the variant sweep: lanes take the bins to solve in
// rank order (1) or bin = lane + 32 * round (0); dAdw in one two-tangent pass (1) or two
// single-tangent passes (0).
#ifndef PZ_BATCHED_RANK
#define PZ_BATCHED_RANK 0
#endif
#ifndef PZ_BATCHED_DADW2
#define PZ_BATCHED_DADW2 1
#endif

constexpr int kWarpsPerBlock = 8;
constexpr int kMaxCand = 96;   // candidate (triangle, segment) entries of one merged query
constexpr int kFront = 128;    // frontier entries per level of the breadth-first query
constexpr float kMaxShift = 0.5f;    // a larger predicted shift over the band falls back
constexpr float kDeep = 0.3f;        // a predicted root this far inside every triangle is refined, not re-solved
constexpr float kProbeTol = 1.0e-3f;  // a plain-solve root farther than this from the followed branch is another root

// Phase-1 result of one work item that has bins to refine (global, compacted).
template <int K> struct PairRec {
    int pixel, slot, mode;  // mode 1: predicted roots, 2: plain per-bin solves
    int polish;             // the item is ill-conditioned: FP64 polish of its roots
    int scene;              // the item's scene in a batch of scenes
    int item;               // the item's index in its scene's work list
    unsigned long long mask;  // bins to solve (mode 1)
    unsigned long long warm;  // of those, bins whose root is deep inside: refine the prediction
    float xa[2 * K], xc[2 * K], xb[2 * K];  // roots at the first, centre and last bin
};

// The plain path's solve of one work item at one probe bin (q = 0: centre, 1: first, 2: last).
template <int K> struct Probe {
    float x[2 * K];
    uint32_t ok;
};

// Quadratic (Lagrange) prediction of the root at eta from the roots at eta_a, eta_c, eta_b.
template <int K>
PZ_D void predict_root(float (&x)[2 * K], const PairRec<K>& r, float eta, float ea, float ec, float eb)
{
    const float la = (eta - ec) * (eta - eb) / ((ea - ec) * (ea - eb));
    const float lc = (eta - ea) * (eta - eb) / ((ec - ea) * (ec - eb));
    const float lb = (eta - ea) * (eta - ec) / ((eb - ea) * (eb - ec));
#pragma unroll
    for (int i = 0; i < 2 * K; i++) x[i] = r.xa[i] * la + r.xc[i] * lc + r.xb[i] * lb;
}

PZ_D float warp_max(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xFFFFFFFFu, v, o));
    return v;
}

// Admissibility part of contributableThroughput<K> (pk.h:769-827); returns 0 if
// rejected, else the Fresnel product; fills the chain vertices and normals used by the
// visibility segments.
template <class T, int K>
PZ_D T pre_throughput(const T* x, V3<T> p_beg, V3<T> p_end, const Chain<K>& ch, uint32_t events, T eta,
                      float3 (&vtx)[K + 2], float3 (&nrm)[K + 2])
{
    V3<T> v[K + 2], sn[K + 2];
    v[0] = p_beg;
    v[K + 1] = p_end;
#pragma unroll
    for (int k = 0; k < K; k++) {
        const T u = x[2 * k], w = x[2 * k + 1];
        if (u < T(0) || w < T(0) || T(1) < u + w) return T(0);
        v[k + 1] = vertex<T, K>(ch, x, k);
        sn[k + 1] = vnormalize(v3f<T>(ch.n0[k]) + v3f<T>(ch.ne0[k]) * u + v3f<T>(ch.ne1[k]) * w);
    }
    sn[0] = vnormalize(v[1] - v[0]);
    sn[K + 1] = vnormalize(v[K] - v[K + 1]);
    T thr = T(1);
#pragma unroll
    for (int k = 0; k < K; k++) {
        const V3<T> wi = v[k] - v[k + 1], wo = v[k + 2] - v[k + 1], n = sn[k + 1];
        const bool eR = T(0) < vdot(wi, n) * vdot(wo, n);
        if (((events >> k) & 1u) == (eR ? 1u : 0u)) return T(0);
        const V3<T> ng = v3f<T>(ch.ng[k]);
        if (eR != (T(0) < vdot(wi, ng) * vdot(wo, ng))) return T(0);
        if (ch.material[k] == kDielectric) {
            const T r = fresnel_T(wi, n, eta);
            thr *= eR ? r : T(1) - r;
        }
    }
#pragma unroll
    for (int i = 0; i < K + 1; i++) {
        const V3<T> d = v[i] - v[i + 1];
        if (vdot(d, d) < T(1.0e-5f)) return T(0);
    }
#pragma unroll
    for (int i = 0; i < K + 2; i++) {
        vtx[i] = mk3((float)v[i].x, (float)v[i].y, (float)v[i].z);
        nrm[i] = mk3((float)sn[i].x, (float)sn[i].y, (float)sn[i].z);
    }
    return thr;
}

// Chain vertex i (0 = light, K + 1 = receiver point) and its normal as
// contributableThroughput builds them (pk.h:763-789), from the barycentrics.
template <int K>
PZ_D void chain_vertex(const Chain<K>& ch, const float* x, float3 p_light, float3 p_end, int i, float3& v, float3& n)
{
    auto vert = [&](int j) -> float3 {
        if (j == 0) return p_light;
        if (j == K + 1) return p_end;
        const V3<float> q = vertex<float, K>(ch, x, j - 1);
        return mk3(q.x, q.y, q.z);
    };
    v = vert(i);
    if (i == 0) {
        n = normalize(vert(1) - vert(0));
    } else if (i == K + 1) {
        n = normalize(vert(K) - vert(K + 1));
    } else {
        const float u = x[2 * (i - 1)], w = x[2 * (i - 1) + 1];
        const V3<float> sn = vnormalize(v3f<float>(ch.n0[i - 1]) + v3f<float>(ch.ne0[i - 1]) * u +
                                        v3f<float>(ch.ne1[i - 1]) * w);
        n = mk3(sn.x, sn.y, sn.z);
    }
}

// a[i] by selects (no stack frame for a runtime index)
template <int N>
PZ_D float3 pick(const float3 (&a)[N], int i)
{
    float3 r = a[0];
#pragma unroll
    for (int j = 1; j < N; j++)
        if (i == j) r = a[j];
    return r;
}

// The shadow-ray segment of occluded() (pk.h:88-115): start and end points.
PZ_D void shadow_segment(float3 from, float3 from_n, float3 to, float3 to_n, float3& a, float3& b)
{
    if (ex::dot(ex::sub3(to, from), from_n) < 0.0f) from_n = -from_n;
    if (ex::dot(ex::sub3(from, to), to_n) < 0.0f) to_n = -to_n;
    a = ex::add3(from, ex::mul3(from_n, ray_offset_scale(from)));
    b = ex::add3(to, ex::mul3(to_n, ray_offset_scale(to)));
}

// Warp-cooperative query of NS segments at once: for each segment s, the leaves whose box,
// grown by r[s], meets the segment [a[s], a[s] + d[s]], found breadth first.  Frontier
// entries are (node, segment) pairs, so the lanes test the frontier nodes of every segment
// side by side, one tree level per step: the chain of dependent node loads is the tree's
// depth, and the frontier of one level holds the nodes of all segments (a frontier of a single
// fattened segment is a few nodes wide, and left most lanes idle).  Leaves that pass are
// appended to the candidate list as (triangle, segment) entries in ballot order, internal
// children to the next level's frontier (two halves of `front`, kFront entries each); a leaf
// is a candidate when its box, and every ancestor's, meets the fattened segment.  Entries
// carry the segment in bits 29-31 (node and triangle indices below 2^29).  Returns the count,
// or -1 when the candidate list or the frontier overflows.
constexpr uint32_t kSegShift = 29;
constexpr uint32_t kIdxMask = (1u << kSegShift) - 1u;

template <int NS>
PZ_D float3 pick3(const float3 (&v)[NS], uint32_t i)
{
    float3 r = v[0];
#pragma unroll
    for (int j = 1; j < NS; j++)
        if (i == (uint32_t)j) r = v[j];
    return r;
}
template <int NS>
PZ_D float pick1(const float (&v)[NS], uint32_t i)
{
    float r = v[0];
#pragma unroll
    for (int j = 1; j < NS; j++)
        if (i == (uint32_t)j) r = v[j];
    return r;
}

template <int NS>
PZ_D int fat_query_multi(const Node* __restrict__ nodes, uint32_t root, const float3 (&a)[NS], const float3 (&inv)[NS],
                         const float (&r)[NS], uint32_t segMask, uint32_t* cand, uint32_t* front)
{
    const int lane = threadIdx.x & 31;
    const uint32_t lt = (1u << lane) - 1u;
    if (root == kInvalidNode || !segMask) return 0;
    if (is_leaf(root)) {
        int n = 0;
#pragma unroll
        for (int s = 0; s < NS; s++)
            if ((segMask >> s) & 1u) {
                if (lane == 0) cand[n] = node_idx(root) | ((uint32_t)s << kSegShift);
                n++;
            }
        return n;
    }
    int nf = 0;
#pragma unroll
    for (int s = 0; s < NS; s++)
        if ((segMask >> s) & 1u) {
            if (lane == 0) front[nf] = node_idx(root) | ((uint32_t)s << kSegShift);
            nf++;
        }
    __syncwarp();
    int n = 0, cur = 0;
    while (nf > 0) {
        int nNext = 0;
        for (int base = 0; base < nf; base += 32) {
            bool hl = false, hr = false;
            uint32_t c0 = 0, c1 = 0, seg = 0;
            if (base + lane < nf) {
                const uint32_t e = front[cur * kFront + base + lane];
                seg = e >> kSegShift;
                const NodeView nv = load_node(nodes, e & kIdxMask);
                const float3 sa = pick3<NS>(a, seg), si = pick3<NS>(inv, seg);
                const float rr = pick1<NS>(r, seg);
                const float3 R = mk3(rr, rr, rr);
                float tl, tr;
                hl = slab_hit(sa, si, nv.lo0 - R, nv.hi0 + R, 1.0f, &tl);
                hr = slab_hit(sa, si, nv.lo1 - R, nv.hi1 + R, 1.0f, &tr);
                c0 = nv.c0;
                c1 = nv.c1;
            }
            const uint32_t tag = seg << kSegShift;
            const uint32_t leaf0 = __ballot_sync(0xFFFFFFFFu, hl && is_leaf(c0));
            const uint32_t leaf1 = __ballot_sync(0xFFFFFFFFu, hr && is_leaf(c1));
            const uint32_t in0 = __ballot_sync(0xFFFFFFFFu, hl && !is_leaf(c0));
            const uint32_t in1 = __ballot_sync(0xFFFFFFFFu, hr && !is_leaf(c1));
            const int nLeaf = __popc(leaf0) + __popc(leaf1), nIn = __popc(in0) + __popc(in1);
            if (n + nLeaf > kMaxCand || nNext + nIn > kFront) return -1;
            uint32_t* next = front + (cur ^ 1) * kFront;
            if ((leaf0 >> lane) & 1u) cand[n + __popc(leaf0 & lt)] = node_idx(c0) | tag;
            if ((leaf1 >> lane) & 1u) cand[n + __popc(leaf0) + __popc(leaf1 & lt)] = node_idx(c1) | tag;
            if ((in0 >> lane) & 1u) next[nNext + __popc(in0 & lt)] = node_idx(c0) | tag;
            if ((in1 >> lane) & 1u) next[nNext + __popc(in0) + __popc(in1 & lt)] = node_idx(c1) | tag;
            n += nLeaf;
            nNext += nIn;
        }
        __syncwarp();
        cur ^= 1;
        nf = nNext;
    }
    return n;
}

// FP64 polish of an ill-conditioned root (kept out of line: rare, register-hungry).
template <int K>
__device__ __noinline__ float polish_fp64(float* xs, const Chain<K>& ch, float3 p_light, float3 p, uint32_t events,
                                          float eta, float3 (&vtx)[K + 2], float3 (&nrm)[K + 2])
{
    double xd[2 * K];
#pragma unroll
    for (int i = 0; i < 2 * K; i++) xd[i] = xs[i];
    const V3<double> Ld = v3f<double>(p_light), pd = v3f<double>(p);
    int itd;
    double detd;
    const bool ok = newton<double, K>(xd, Ld, pd, ch, (double)eta, events, 4, 1.0e-24, 0, false, &itd, &detd);
    // keep the polished root only if it converged next to the FP32 root
    double moved = 0.0;
#pragma unroll
    for (int i = 0; i < 2 * K; i++) moved = fmax(moved, fabs(xd[i] - (double)xs[i]));
    if (!ok || !(moved < 1.0e-3)) {
        const V3<float> L = v3f<float>(p_light);
        return pre_throughput<float, K>(xs, L, v3f<float>(p), ch, events, eta, vtx, nrm);
    }
    const double t = pre_throughput<double, K>(xd, Ld, pd, ch, events, (double)eta, vtx, nrm);
#pragma unroll
    for (int i = 0; i < 2 * K; i++) xs[i] = (float)xd[i];
    return (float)t;
}

// Smallest |cos| between a path segment and the shading normal over the chain's vertices
// at the root x (the path grazes a surface when it is small).
template <int K>
__device__ __noinline__ float min_abs_cos(const Chain<K>& ch, const float* x, float3 p_light, float3 p)
{
    float m = 1.0f;
#pragma unroll
    for (int k = 1; k <= K; k++) {
        float3 va, na, v, n, vb, nb;
        chain_vertex<K>(ch, x, p_light, p, k - 1, va, na);
        chain_vertex<K>(ch, x, p_light, p, k, v, n);
        chain_vertex<K>(ch, x, p_light, p, k + 1, vb, nb);
        m = fminf(m, fabsf(dot(normalize(va - v), n)));
        m = fminf(m, fabsf(dot(normalize(vb - v), n)));
    }
    return m;
}

template <int K>
__device__ __noinline__ float dadw_out_of_line(const Chain<K>& ch, const float* xs, float3 p_light, float3 p,
                                               uint32_t events, float eta)
{
    const V3<float> L = v3f<float>(p_light);
    const V3<float> v0 = vertex<float, K>(ch, xs, 0);
#if PZ_BATCHED_DADW2
    return dadw2<float, K>(L, v0 - L, v3f<float>(p), ch, events, eta);
#else
    return dadw<float, K>(L, v0 - L, v3f<float>(p), ch, events, eta);
#endif
}

// Newton on the multi-tangent Jacobian, out of line: one copy of the body serves every
// call site (the kernels are instruction-cache bound when it is inlined several times).
template <int K>
__device__ __noinline__ bool newton_nl(float* x, const Chain<K>& ch, float3 p_light, float3 p, float eta,
                                       uint32_t events, int maxIterations, float tol, int warmup, bool edge,
                                       int minSteps, float* det, int* itersOut = nullptr)
{
    int it;
    const bool c = newton<float, K>(x, v3f<float>(p_light), v3f<float>(p), ch, eta, events, maxIterations, tol, warmup,
                                    edge, &it, det, minSteps);
    if (itersOut) *itersOut = it;
    return c;
}

// The plain path's solve (solveConstraints' rules from the photon's start: cost tolerance,
// edge rejection after the warm-up iterations) on the multi-tangent Jacobian, whose
// columns follow the reference's single-tangent operation order.  Out of line: phase 2
// calls it for every bin that is not refined from a prediction.
template <int K>
__device__ __noinline__ bool plain_solve(float* x, const Chain<K>& ch, float3 p_light, float3 p, float eta,
                                         uint32_t events, int maxIterations, float tol, int warmup)
{
    float det;
    return newton_nl<K>(x, ch, p_light, p, eta, events, maxIterations, tol, warmup, true, 0, &det);
}

// ---------------------------------------------------------------- scenes of a batch
// A work item's scene: the single scene of the call, or, for a batch of scenes, the one
// whose range of the concatenated item list holds it (offsets[s] <= idx < offsets[s + 1]).
struct SceneRef {
    const SolveArgs* s;
    uint64_t local;
    uint32_t scene;
};
template <bool kMulti>
PZ_D SceneRef item_scene(const BatchArgs& a, uint64_t idx)
{
    if (!kMulti) return SceneRef{&a.s, idx, 0u};
    uint32_t lo = 0, hi = a.nScenes;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (a.offsets[mid] <= idx) lo = mid;
        else hi = mid;
    }
    return SceneRef{&a.scenes[lo].s, idx - a.offsets[lo], lo};
}
template <bool kMulti>
PZ_D uint64_t total_items(const BatchArgs& a)
{
    if (kMulti) return a.offsets[a.nScenes];
    return a.nPathsDev ? min((uint64_t)*a.nPathsDev, a.s.nPaths) : a.s.nPaths;
}

// Item offsets of a batch of scenes: exclusive scan of each scene's item count (its
// device counter, capped at its capacity).  One block.
__global__ void k_scene_offsets(const SceneArgs* scenes, uint32_t n, unsigned long long* offsets)
{
    __shared__ unsigned long long carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (uint32_t base = 0; base < n; base += blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        unsigned long long c = 0;
        if (i < n) {
            const SceneArgs& sa = scenes[i];
            c = sa.nPathsDev ? min((uint64_t)*sa.nPathsDev, sa.s.nPaths) : sa.s.nPaths;
        }
        // block-wide inclusive scan (Hillis-Steele in shared memory)
        __shared__ unsigned long long buf[1024];
        buf[threadIdx.x] = c;
        __syncthreads();
        for (uint32_t o = 1; o < blockDim.x; o <<= 1) {
            const unsigned long long v = threadIdx.x >= o ? buf[threadIdx.x - o] : 0ull;
            __syncthreads();
            buf[threadIdx.x] += v;
            __syncthreads();
        }
        if (i < n) offsets[i] = carry + buf[threadIdx.x] - c;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry += buf[threadIdx.x];
        __syncthreads();
    }
    if (threadIdx.x == 0) offsets[n] = carry;
}

// ---------------------------------------------------------------- probes
// One thread per (work item, probe bin): the plain path's solver from the photon's start at
// the centre, first and last bin.  Kept apart from phase 1 so that it runs at the plain
// kernel's occupancy; the three probes of an item sit in adjacent threads.
template <int K, bool kMulti>
__global__ void __launch_bounds__(256) k_probe(BatchArgs a)
{
    const int B = a.s.nBins;
    const uint64_t nPaths = total_items<kMulti>(a);
    auto* probes = reinterpret_cast<Probe<K>*>(a.probes);
    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < 3 * nPaths;
         t += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t idx = t / 3;
        const int q = (int)(t - 3 * idx);
        const SceneRef R = item_scene<kMulti>(a, idx);
        const SolveArgs& S = *R.s;
        const V3<float> L = v3f<float>(S.p_light);
        const SpecularPath sp = S.paths[R.local];
        const int4 ti = S.cache.tris[sp.cacheIndex];
        const int tix[4] = {ti.x, ti.y, ti.z, ti.w};
        Chain<K> ch;
        load_chain<K>(ch, S.tris, S.attribs, tix);
        const float4 q0 = S.cache.params[2 * sp.cacheIndex], q1 = S.cache.params[2 * sp.cacheIndex + 1];
        const float pp[8] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
        Probe<K> r;
#pragma unroll
        for (int i = 0; i < 2 * K; i++) r.x[i] = pp[i];
        const int b = q == 0 ? B / 2 : (q == 1 ? 0 : B - 1);
        float det;
        r.ok = newton_nl<K>(r.x, ch, S.p_light, S.fds[sp.pixel].p, S.etas[b], S.events, S.maxIterations,
                            S.costTolerance, S.earlyTermWarmUp, true, 0, &det)
                   ? 1u
                   : 0u;
        probes[t] = r;
    }
}

// ---------------------------------------------------------------- phase 1
// Adds a per-thread count to a diagnostic counter: a warp sum, then one atomic per warp.
// Called by all 32 lanes after the kernels' loops.
PZ_D void flush_count(unsigned long long* counter, unsigned long long v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(counter, v);
}

#ifndef PZ_PHASE1_PROBE_START
#define PZ_PHASE1_PROBE_START 1
#endif

template <int K, bool kMulti>
__global__ void __launch_bounds__(256, kPhase1Blocks) k_phase1(BatchArgs a)
{
    const int B = a.s.nBins;
    const uint64_t nPaths = total_items<kMulti>(a);
    const int bc = B / 2;
    auto* recs = reinterpret_cast<PairRec<K>*>(a.records);
    unsigned long long nItems = 0;
    // diagnostic counts, kept per thread and added once at the end
    unsigned long long cMode0 = 0, cMode1 = 0, cMode2 = 0, cProbe = 0, cShift = 0, cNoConv = 0, cFold = 0;
    for (uint64_t idx = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < nPaths;
         idx += (uint64_t)gridDim.x * blockDim.x) {
        const SceneRef R = item_scene<kMulti>(a, idx);
        const SolveArgs& S = *R.s;
        const float eta_c = S.etas[bc];
        const V3<float> L = v3f<float>(S.p_light);
        const SpecularPath sp = S.paths[R.local];
        const int4 ti = S.cache.tris[sp.cacheIndex];
        const int tix[4] = {ti.x, ti.y, ti.z, ti.w};
        Chain<K> ch;
        load_chain<K>(ch, S.tris, S.attribs, tix);
        const float4 q0 = S.cache.params[2 * sp.cacheIndex], q1 = S.cache.params[2 * sp.cacheIndex + 1];
        const float pp[8] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
        float x[2 * K], xpc[2 * K];
#pragma unroll
        for (int i = 0; i < 2 * K; i++) x[i] = xpc[i] = pp[i];
        const V3<float> p = v3f<float>(S.fds[sp.pixel].p);
        float det = 1.0f;
        // the plain path's decision at the centre bin (k_probe); when it converged, its root
        // is the branch followed below
        const auto* pr = reinterpret_cast<const Probe<K>*>(a.probes) + 3 * idx;
        const bool okc = pr[0].ok != 0;
#pragma unroll
        for (int i = 0; i < 2 * K; i++) xpc[i] = pr[0].x[i];
        bool conv = okc;
        if (okc) {
#pragma unroll
            for (int i = 0; i < 2 * K; i++) x[i] = xpc[i];
        } else {
#if PZ_PHASE1_PROBE_START
            // the centre probe's last iterate (two Newton steps from the photon's start, where
            // its edge test stopped it) starts the unconstrained solve, when it is finite
            bool usable = true;
#pragma unroll
            for (int i = 0; i < 2 * K; i++) usable = usable && fabsf(xpc[i]) < 1.0e3f;
            if (usable) {
#pragma unroll
                for (int i = 0; i < 2 * K; i++) x[i] = xpc[i];
            }
#endif
            conv = newton_nl<K>(x, ch, S.p_light, S.fds[sp.pixel].p, eta_c, S.events, 24, S.costTolerance, 0, false, 0,
                                &det);
        }
        PairRec<K> r;
        r.pixel = sp.pixel;
        r.slot = sp.cacheIndex;
        r.scene = (int)R.scene;
        r.item = (int)R.local;
        r.mode = 2;
        r.polish = 0;
        r.mask = 0;
        r.warm = 0;
        bool conv2 = false, probeFallback = false;
        if (conv && B >= 3) {
            // root derivative in eta at the centre (implicit-function theorem) and the two
            // end-bin roots, warm-started from the tangent prediction
            float J[2 * K + 1][3 * K], c[3 * K], cost;
            eval_constraints<float, K, true>(x, L, p, ch, eta_c, S.events, J, c, cost);
            float Jx[2 * K][3 * K], rhs[3 * K], dxe[2 * K];
#pragma unroll
            for (int i = 0; i < 2 * K; i++)
#pragma unroll
                for (int j = 0; j < 3 * K; j++) Jx[i][j] = J[i][j];
#pragma unroll
            for (int j = 0; j < 3 * K; j++) rhs[j] = J[2 * K][j];
            det = qr_solve_reldet<float, 3 * K, 2 * K>(Jx, rhs, dxe);
            const float ea = S.etas[0], eb = S.etas[B - 1];
            float lin_a[2 * K], lin_b[2 * K];
#pragma unroll
            for (int i = 0; i < 2 * K; i++) {
                r.xc[i] = x[i];
                lin_a[i] = x[i] - (ea - eta_c) * dxe[i];
                lin_b[i] = x[i] - (eb - eta_c) * dxe[i];
                r.xa[i] = lin_a[i];
                r.xb[i] = lin_b[i];
            }
            float da, db;
            const bool ca =
                newton_nl<K>(r.xa, ch, S.p_light, S.fds[sp.pixel].p, ea, S.events, 12, S.costTolerance, 0, false, 1, &da);
            const bool cb =
                newton_nl<K>(r.xb, ch, S.p_light, S.fds[sp.pixel].p, eb, S.events, 12, S.costTolerance, 0, false, 1, &db);
            float nonlin = 0.0f;
            bool finite = true;
#pragma unroll
            for (int i = 0; i < 2 * K; i++) {
                nonlin = fmaxf(nonlin, fmaxf(fabsf(r.xa[i] - lin_a[i]), fabsf(r.xb[i] - lin_b[i])));
                finite = finite && fabsf(r.xa[i]) < 1.0e6f && fabsf(r.xb[i]) < 1.0e6f && fabsf(x[i]) < 1.0e6f;
            }
            const float minDet = fminf(det, fminf(da, db));
            conv2 = ca && cb;
            if (minDet < a.illDet) {
                // near a fold of the root curve: plain per-bin solves, FP64 polish when near-singular
                r.polish = (double)minDet < a.polishDet ? 1 : 0;
                cFold++;
            } else if (ca && cb && finite && nonlin < kMaxShift) {
                // A bin contributes only if its root lies inside every triangle, so a bin whose
                // predicted root is outside by more than the prediction error cannot contribute.
                const float err = 2.0f * nonlin + 1.0e-4f;
                unsigned long long mask = 0, warm = 0;
                for (int b = 0; b < B; b++) {
                    float xp[2 * K];
                    predict_root<K>(xp, r, S.etas[b], ea, eta_c, eb);
                    float depth = 1.0f;
#pragma unroll
                    for (int k = 0; k < K; k++)
                        depth = fminf(depth, fminf(fminf(xp[2 * k], xp[2 * k + 1]), 1.0f - xp[2 * k] - xp[2 * k + 1]));
                    if (depth > -err) mask |= 1ull << b;
                    if (depth > kDeep + err) warm |= 1ull << b;
                }
                // the bin next to each end of a contributing run is solved too: that is where a
                // root crosses a triangle edge, and where the prediction error matters most
                const unsigned long long all = B == 64 ? ~0ull : ((1ull << B) - 1ull);
                mask = (mask | (mask << 1) | (mask >> 1)) & all;
                r.mask = mask;
                r.warm = warm;
                r.mode = mask ? 1 : 0;
                // The plain path solves every bin from the photon's start, so its root can lie on
                // another branch than the one followed here.  Probe the plain solve at the
                // centre and both end bins: a converged root away from the followed branch, or a
                // rejection where the branch is deep inside, sends the item to per-bin plain solves.
                bool mismatch = false;
#pragma unroll 1
                for (int q = 0; q < 3 && !mismatch; q++) {
                    const int b = q == 0 ? bc : (q == 1 ? 0 : B - 1);
                    const float* xt = q == 0 ? r.xc : (q == 1 ? r.xa : r.xb);
                    float xq[2 * K];
                    const bool okq = pr[q].ok != 0;
#pragma unroll
                    for (int i = 0; i < 2 * K; i++) xq[i] = pr[q].x[i];
                    if (okq) {
                        float dev = 0.0f;
#pragma unroll
                        for (int i = 0; i < 2 * K; i++) dev = fmaxf(dev, fabsf(xq[i] - xt[i]));
                        mismatch = !(dev < kProbeTol);
                    } else {
                        mismatch = ((warm >> b) & 1ull) != 0;
                    }
                }
                if (mismatch) {
                    probeFallback = true;
                    r.mode = 2;
                    r.mask = 0;
                    r.warm = 0;
                    cProbe++;
                }
            }
        }
        nItems += (unsigned long long)B;
        cMode0 += r.mode == 0;
        cMode1 += r.mode == 1;
        cMode2 += r.mode == 2;
        if (r.mode == 2 && !probeFallback) {
            cShift += conv && conv2;
            cNoConv += !(conv && conv2);
        }
        // warp-aggregated appends of the items that have work: predicted items from the front
        // of the records array, items solved bin by bin from its end
        const bool keep1 = r.mode == 1, keep2 = r.mode == 2;
        const uint32_t active = __activemask();
        const uint32_t lt = (1u << (threadIdx.x & 31)) - 1u;
        const uint32_t b1 = __ballot_sync(active, keep1), b2 = __ballot_sync(active, keep2);
        const int leader = __ffs(active) - 1;
        unsigned long long s1 = 0, s2 = 0;
        if ((int)(threadIdx.x & 31) == leader) {
            if (b1) s1 = atomicAdd(a.recordCount, (unsigned long long)__popc(b1));
            if (b2) s2 = atomicAdd(a.recordCount2, (unsigned long long)__popc(b2));
        }
        s1 = __shfl_sync(active, s1, leader);
        s2 = __shfl_sync(active, s2, leader);
        if (keep1) {
            const unsigned long long dst = s1 + __popc(b1 & lt);
            if (dst < a.recordCapacity) recs[dst] = r;
            else raise_error(a.status, kErrCapacity);
        }
        if (keep2) {
            const unsigned long long k = s2 + __popc(b2 & lt);
            if (k < a.recordCapacity) recs[a.recordCapacity - 1 - k] = r;
            else raise_error(a.status, kErrCapacity);
        }
    }
    if (a.s.stats) flush_count(a.s.stats + 0, nItems);
    if (a.counters) {
        flush_count(a.counters + kCntMode0, cMode0);
        flush_count(a.counters + kCntMode1, cMode1);
        flush_count(a.counters + kCntMode2, cMode2);
        flush_count(a.counters + kCntFallbackProbe, cProbe);
        flush_count(a.counters + kCntFallbackShift, cShift);
        flush_count(a.counters + kCntFallbackNoConv, cNoConv);
        flush_count(a.counters + kCntFallbackFold, cFold);
    }
}

// ---------------------------------------------------------------- phase 2
// Phase 2 runs in waves of three kernels.  Each wave takes records (phase-1 items with bins
// to solve) from the work counter while the accepted list has room for B more roots per
// record (a record never has more), so any input fits in a fixed number of waves:
//  * k_p2_solve, persistent warps: the 32 lanes of a round take (record, bin) pairs, the
//    bins of a record in rank order on consecutive lanes (a record solved bin by bin starts
//    a round; predicted records are packed one after another); Newton, then
//    admissibility; the accepted (converged and admissible) roots of a record leave as one
//    block {first, record, count} (a per-warp stash joins the roots of a record split
//    between two rounds);
//  * k_p2_vis, one warp per block: the shadow segments of the block's roots share one
//    fattened BVH query per path segment (all roots of a block belong to one record, so
//    their segments are close); a root that is occluded gets throughput 0;
//  * k_p2_contrib, one thread per accepted root: dAdw and the clamped contribution, added
//    to the spectral image.
// Each kernel is a short body at modest register count, where the single phase-2 kernel it
// replaces held Newton, the queries and dAdw at once (instruction-fetch bound at 25%
// occupancy, and idle lanes for every bin a record did not solve).

// Accepted root of phase 2.
template <int K> struct Accepted {
    uint32_t rec;   // phase-1 record
    uint32_t bin;   // wavelength bin
    float thr;      // Fresnel product after admissibility; 0 once occluded
    float x[2 * K]; // barycentrics of the root
};
// Round of accepted roots of one record: entries [first, first + count) of the accepted list.
struct AcceptBlock {
    uint32_t first, rec, count;
};

// The record's bin mask to solve.
template <int K>
PZ_D unsigned long long record_todo(const PairRec<K>& r, int B)
{
    return r.mode == 2 ? (B == 64 ? ~0ull : ((1ull << B) - 1ull)) : r.mask;
}

// m without its n lowest set bits.
PZ_D unsigned long long drop_low_bits(unsigned long long m, int n)
{
    if (n >= __popcll(m)) return 0ull;
    const int p = nth_bit64(m, n);
    return m & ~((1ull << p) - 1ull);
}

template <int K, bool kMulti>
__global__ void __launch_bounds__(kWarpsPerBlock * 32, kP2SolveBlocks) k_p2_solve(BatchArgs a)
{
    const int lane = threadIdx.x & 31;
    const uint32_t lt = (1u << lane) - 1u;
    const int B = a.s.nBins;
    // The records solved bin by bin (the second queue) come first, then the predicted ones:
    // one index space [0, nRec2 + nRec1) on one work counter, so a wave stops taking records
    // only when its accepted list is full or every record is taken.
    const unsigned long long nRec2 = min(*a.recordCount2, a.recordCapacity);
    const unsigned long long nRec = nRec2 + min(*a.recordCount, a.recordCapacity);
    const auto* recs = reinterpret_cast<const PairRec<K>*>(a.records);
    auto* acc = reinterpret_cast<Accepted<K>*>(a.accepted);
    auto* blocks = reinterpret_cast<AcceptBlock*>(a.blocks);
    unsigned long long* const nAccepted = a.p2 + 0;
    unsigned long long* const nBlocks = a.p2 + 1;
    unsigned long long* const reserved = a.p2 + 2;
    unsigned long long nConv = 0, cNewton = 0, cPolish = 0, cIters = 0, cWarm = 0;
    // The warp's current record and the bins of it not yet handed to a lane, and the records
    // it has claimed and not yet started, [jNext, jEnd) (all warp-uniform).
    unsigned long long jc = 0, mc = 0, jNext = 0, jEnd = 0;
    bool drained = false;
    const unsigned long long chunk = (unsigned long long)(a.chunk > 0 ? a.chunk : kP2ChunkDefault);
    // accepted roots held back for the next round: ns entries of record stashRec
    __shared__ Accepted<K> stash[kWarpsPerBlock][32];
    const int warp = threadIdx.x >> 5;
    int ns = 0;
    unsigned long long stashRec = 0;
    for (;;) {
        // Fill the 32 lanes with (record, bin) pairs.  A record solved bin by bin (every bin
        // from the photon's start) starts a round, or joins one only if all its bins fit, so
        // the bins of a round mostly share one chain and one start and follow similar Newton
        // paths.  A predicted record is packed: its bins in rank order, then the next
        // record's, so no lane idles for a bin that a record's mask excludes.  Records are
        // claimed `chunk` at a time (one atomic each on the work counter and on the room
        // reserved for B accepted roots per record, a record's most, in this wave).
        int filled = 0;
        unsigned long long myRec = 0;
        int myBin = -1;
        while (filled < 32) {
            if (mc == 0) {
                if (jNext == jEnd) {
                    if (drained) break;
                    unsigned long long j = 0, cnt = 0;
                    if (lane == 0) {
                        const unsigned long long room = (unsigned long long)B * chunk;
                        if (*a.workCounter < nRec && atomicAdd(reserved, room) + room <= a.acceptCapacity) {
                            j = atomicAdd(a.workCounter, chunk);
                            cnt = j < nRec ? min(chunk, nRec - j) : 0ull;
                        }
                    }
                    cnt = __shfl_sync(0xFFFFFFFFu, cnt, 0);
                    if (cnt == 0) {
                        drained = true;
                        break;
                    }
                    jNext = __shfl_sync(0xFFFFFFFFu, j, 0);
                    jEnd = jNext + cnt;
                }
                const bool whole = jNext < nRec2;
                if (whole && filled != 0 && B > 32 - filled) break;  // it starts the next round
                jc = whole ? a.recordCapacity - 1 - jNext : jNext - nRec2;
                jNext++;
                mc = record_todo<K>(recs[jc], B);
                continue;
            }
            const int n = min(__popcll(mc), 32 - filled);
            if (lane >= filled && lane < filled + n) {
                myRec = jc;
                myBin = nth_bit64(mc, lane - filled);
            }
            mc = drop_low_bits(mc, n);
            filled += n;
        }
        if (filled == 0) break;
        float xs[2 * K];
        float thr = 0.0f;
        if (myBin >= 0) {
            const int b = myBin;
            const PairRec<K> r = recs[myRec];
            const SolveArgs& S = kMulti ? a.scenes[r.scene].s : a.s;
            const float eta_c = S.etas[B / 2];
            const V3<float> L = v3f<float>(S.p_light);
            const int4 ti = S.cache.tris[r.slot];
            const int tix[4] = {ti.x, ti.y, ti.z, ti.w};
            Chain<K> ch;
            load_chain<K>(ch, S.tris, S.attribs, tix);
            const float3 pe = S.fds[r.pixel].p;
            const V3<float> p = v3f<float>(pe);
            const float eta = S.etas[b];
            const bool warm = r.mode == 1 && (a.continuation || ((r.warm >> b) & 1ull));
            if (warm) {
                predict_root<K>(xs, r, eta, S.etas[0], eta_c, S.etas[B - 1]);
            } else {
                const float4 q0 = S.cache.params[2 * r.slot], q1 = S.cache.params[2 * r.slot + 1];
                const float pp[8] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
#pragma unroll
                for (int i = 0; i < 2 * K; i++) xs[i] = pp[i];
            }
            float det = 1.0f;
            int its = 0;
            // a predicted root is refined by Newton; every other bin runs the plain path's
            // solver from the photon's start, so its accept / reject decision is the plain one
            const bool conv = newton_nl<K>(xs, ch, S.p_light, pe, eta, S.events, S.maxIterations, S.costTolerance,
                                           S.earlyTermWarmUp, true, warm ? 1 : 0, &det, &its);
            cNewton++;
            cIters += its;
            cWarm += warm;
            if (conv && S.roots) {
                float* rt = S.roots + ((size_t)r.item * B + b) * 8;
#pragma unroll
                for (int i = 0; i < 2 * K; i++) rt[i] = xs[i];
            }
            if (conv) {
                nConv++;
                const bool polish = r.polish || (double)det < a.polishDet ||
                                    (a.grazeCos > 0.0f && min_abs_cos<K>(ch, xs, S.p_light, pe) < a.grazeCos);
                cPolish += polish;
                float3 vtx[K + 2], nrm[K + 2];
                if (polish)
                    thr = polish_fp64<K>(xs, ch, S.p_light, pe, S.events, eta, vtx, nrm);
                else
                    thr = pre_throughput<float, K>(xs, L, p, ch, S.events, eta, vtx, nrm);
            }
        }
        // This round's accepted roots, as blocks of consecutive entries, one per record: a
        // record's bins sit on consecutive lanes, so ordering the entries by lane keeps each
        // record's entries together.  The roots of a record that continues into the next round
        // are held in the warp's stash and leave with that record's next roots, so a record
        // split between rounds still makes one block (one shared visibility query) when its
        // roots number 32 or fewer.
        const uint32_t ok = __ballot_sync(0xFFFFFFFFu, thr > 0.0f);
        const bool hasBin = myBin >= 0;
        const uint32_t contMask = mc != 0 ? __ballot_sync(0xFFFFFFFFu, hasBin && myRec == jc) : 0u;
        const uint32_t g0Mask = ns > 0 ? __ballot_sync(0xFFFFFFFFu, hasBin && myRec == stashRec) : 0u;
        const uint32_t okS = ok & contMask, okE = ok & ~contMask;
        const uint32_t g0E = okE & g0Mask;
        bool emitStash = false, merged = false;
        int keep = 0;
        if (ns > 0) {
            if ((g0Mask & contMask) != 0) {
                // the stashed record continues once more
                if (ns + __popc(okS) > 32) emitStash = true;
                else keep = ns;
            } else {
                emitStash = true;
                merged = ns + __popc(g0E) <= 32;
            }
        }
        Accepted<K> e;
        e.rec = (uint32_t)myRec;
        e.bin = (uint32_t)myBin;
        e.thr = thr;
#pragma unroll
        for (int i = 0; i < 2 * K; i++) e.x[i] = xs[i];
        const int sOut = emitStash ? ns : 0;
        const uint32_t grp = __match_any_sync(0xFFFFFFFFu, hasBin ? myRec : ~0ull) & okE;
        const bool leader = grp != 0 && lane == __ffs(grp) - 1 && !(merged && ((g0Mask >> lane) & 1u));
        const uint32_t leaders = __ballot_sync(0xFFFFFFFFu, leader);
        const int nOut = sOut + __popc(okE);
        if (nOut > 0) {
            unsigned long long first = 0, bi0 = 0;
            if (lane == 0) {
                first = atomicAdd(nAccepted, (unsigned long long)nOut);
                bi0 = atomicAdd(nBlocks, (unsigned long long)((emitStash ? 1 : 0) + __popc(leaders)));
            }
            first = __shfl_sync(0xFFFFFFFFu, first, 0);
            bi0 = __shfl_sync(0xFFFFFFFFu, bi0, 0);
            // the stash's block: its entries, then (merged) the same record's roots of this round
            if (emitStash && lane == 0) {
                const uint32_t cnt = (uint32_t)(ns + (merged ? __popc(g0E) : 0));
                if (bi0 < a.blockCapacity && first + cnt <= a.acceptCapacity)
                    blocks[bi0] = AcceptBlock{(uint32_t)first, (uint32_t)stashRec, cnt};
                else
                    raise_error(a.status, kErrCapacity);  // cannot happen: room was reserved
            }
            if (leader) {
                const unsigned long long bi = bi0 + (emitStash ? 1 : 0) + __popc(leaders & lt);
                const unsigned long long dst = first + sOut + __popc(okE & lt);
                if (bi < a.blockCapacity && dst + __popc(grp) <= a.acceptCapacity)
                    blocks[bi] = AcceptBlock{(uint32_t)dst, (uint32_t)myRec, (uint32_t)__popc(grp)};
                else
                    raise_error(a.status, kErrCapacity);
            }
            if (emitStash && lane < ns && first + lane < a.acceptCapacity) acc[first + lane] = stash[warp][lane];
            if ((okE >> lane) & 1u) {
                const unsigned long long dst = first + sOut + __popc(okE & lt);
                if (dst < a.acceptCapacity) acc[dst] = e;
            }
        }
        __syncwarp();
        if ((okS >> lane) & 1u) stash[warp][keep + __popc(okS & lt)] = e;
        ns = contMask ? keep + __popc(okS) : 0;
        stashRec = jc;
        __syncwarp();
    }
    if (a.s.stats) flush_count(a.s.stats + 1, nConv);
    if (a.counters) {
        flush_count(a.counters + kCntNewton2, cNewton);
        flush_count(a.counters + kCntPolish, cPolish);
        flush_count(a.counters + kCntNewtonIters, cIters);
        flush_count(a.counters + kCntWarm, cWarm);
    }
}

#ifndef PZ_VIS_GROUP
#define PZ_VIS_GROUP 2
#endif
constexpr unsigned long long kVisGroup = PZ_VIS_GROUP;  // blocks a visibility warp claims at once (even)
static_assert(PZ_VIS_GROUP >= 2 && PZ_VIS_GROUP % 2 == 0, "PZ_VIS_GROUP: an even count");

template <int K, bool kMulti>
__global__ void __launch_bounds__(kWarpsPerBlock * 32, 3) k_p2_vis(BatchArgs a)
{
    constexpr int NS = K + 1;
    __shared__ uint32_t cand[kWarpsPerBlock][kMaxCand];
    __shared__ uint32_t front[kWarpsPerBlock][2 * kFront];
    // every root's shadow segments, so that any lane can test any (candidate, root) pair
    // (components apart, so that lanes reading different roots' segments hit different banks)
    __shared__ float segA[kWarpsPerBlock][NS][3][32], segD[kWarpsPerBlock][NS][3][32];
    __shared__ uint32_t occMask[kWarpsPerBlock];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned long long nB = min(a.p2[1], a.blockCapacity);
    // every record is taken by the last wave (each wave takes a fixed share or the rest); a
    // record left over would be a missing contribution, so it is reported
    if (a.wave == kMaxWaves - 1 && blockIdx.x == 0 && threadIdx.x == 0 &&
        *a.workCounter < min(*a.recordCount, a.recordCapacity) + min(*a.recordCount2, a.recordCapacity))
        raise_error(a.status, kErrCapacity);
    const auto* recs = reinterpret_cast<const PairRec<K>*>(a.records);
    auto* acc = reinterpret_cast<Accepted<K>*>(a.accepted);
    const auto* blocks = reinterpret_cast<const AcceptBlock*>(a.blocks);
    unsigned long long cQueries = 0, cOverflow = 0, cCand = 0;
    for (;;) {
        // Blocks are taken in pairs.  Two blocks of one tuple (consecutive records: the work
        // list is in tuple order, so neighbouring pixels) whose roots fit the warp share one
        // query, fattened to cover both; otherwise the warp runs them one after the other.
        unsigned long long bg = 0;
        if (lane == 0) bg = atomicAdd(a.p2 + 3, (unsigned long long)kVisGroup);
        bg = __shfl_sync(0xFFFFFFFFu, bg, 0);
        if (bg >= nB) break;
        for (unsigned long long bi = bg; bi < bg + kVisGroup && bi < nB; bi += 2) {
        const AcceptBlock b0 = blocks[bi];
        const bool has1 = bi + 1 < nB;
        const AcceptBlock b1 = has1 ? blocks[bi + 1] : AcceptBlock{0u, b0.rec, 0u};
        bool merge = false;
        if (has1 && b0.count + b1.count <= 32u) {
            const PairRec<K>& r0 = recs[b0.rec];
            const PairRec<K>& r1 = recs[b1.rec];
            merge = r0.slot == r1.slot && r0.scene == r1.scene;
        }
        const int units = merge ? 1 : (has1 ? 2 : 1);
        for (int unit = 0; unit < units; unit++) {
            // this lane's block and its root's index in it
            AcceptBlock blk = unit == 0 ? b0 : b1;
            uint32_t idx = (uint32_t)lane;
            if (merge && (uint32_t)lane >= b0.count) {
                blk = b1;
                idx = (uint32_t)lane - b0.count;
            }
            const PairRec<K>& r = recs[blk.rec];
            const SolveArgs& S = kMulti ? a.scenes[r.scene].s : a.s;
            const uint32_t root = __ldg(S.root);
            const int4 ti = S.cache.tris[r.slot];
            const int tix[4] = {ti.x, ti.y, ti.z, ti.w};
            Chain<K> ch;
            load_chain<K>(ch, S.tris, S.attribs, tix);
            const float3 pe = S.fds[r.pixel].p;
            const bool mine = idx < blk.count;
            float thr = 0.0f;
            float xs[2 * K];
            if (mine) {
                const Accepted<K>& e = acc[blk.first + idx];
                thr = e.thr;
#pragma unroll
                for (int i = 0; i < 2 * K; i++) xs[i] = e.x[i];
            }
            // the shadow segments of every root: endpoints are the chain's vertices and shading
            // normals (contributableThroughput, pk.h:763-789), offset as occluded() does
            float3 sa[NS], sd[NS];
#pragma unroll
            for (int sg = 0; sg < NS; sg++) sa[sg] = sd[sg] = mk3(0.f, 0.f, 0.f);
            if (thr > 0.0f) {
                float3 va, na;
                chain_vertex<K>(ch, xs, S.p_light, pe, 0, va, na);
#pragma unroll
                for (int sg = 0; sg < NS; sg++) {
                    float3 vb, nb, b;
                    chain_vertex<K>(ch, xs, S.p_light, pe, sg + 1, vb, nb);
                    shadow_segment(va, na, vb, nb, sa[sg], b);
                    sd[sg] = ex::sub3(b, sa[sg]);
                    va = vb;
                    na = nb;
                }
            }
            const uint32_t valid = __ballot_sync(0xFFFFFFFFu, thr > 0.0f);
            if (valid) {
                // one merged query for all segments, each fattened to cover every root's segment
                const int leader = __ffs(valid) - 1;
                float3 ra[NS], rinv[NS];
                float rad[NS];
#pragma unroll
                for (int sg = 0; sg < NS; sg++) {
                    ra[sg] = mk3(__shfl_sync(0xFFFFFFFFu, sa[sg].x, leader), __shfl_sync(0xFFFFFFFFu, sa[sg].y, leader),
                                 __shfl_sync(0xFFFFFFFFu, sa[sg].z, leader));
                    const float3 rd = mk3(__shfl_sync(0xFFFFFFFFu, sd[sg].x, leader),
                                          __shfl_sync(0xFFFFFFFFu, sd[sg].y, leader),
                                          __shfl_sync(0xFFFFFFFFu, sd[sg].z, leader));
                    const float3 rb = ra[sg] + rd;
                    rinv[sg] = inv_rd(rb - ra[sg]);
                    float dev = 0.0f, mag = 0.0f;
                    if (thr > 0.0f) {
                        const float3 da = vabs(sa[sg] - ra[sg]), db = vabs((sa[sg] + sd[sg]) - rb);
                        dev = fmaxf(fmaxf(fmaxf(da.x, da.y), da.z), fmaxf(fmaxf(db.x, db.y), db.z));
                        const float3 ma = vabs(sa[sg]), mb = vabs(sa[sg] + sd[sg]);
                        mag = fmaxf(fmaxf(fmaxf(ma.x, ma.y), ma.z), fmaxf(fmaxf(mb.x, mb.y), mb.z));
                    }
                    // covers the rounding of the slab and box arithmetic
                    rad[sg] = warp_max(dev) + 1.0e-5f * (1.0f + warp_max(mag));
                }
                const int nc = fat_query_multi<NS>(S.nodes, root, ra, rinv, rad, (1u << NS) - 1u, cand[warp], front[warp]);
                __syncwarp();
                if (lane == 0) {
                    cQueries++;
                    if (nc < 0) cOverflow++;
                    else cCand += (unsigned long long)nc;
                }
                if (nc < 0) {
                    // the candidate list overflowed: each root walks the BVH itself
                    bool occ = false;
                    if (thr > 0.0f) {
#pragma unroll 1
                        for (int sg = 0; sg < NS && !occ; sg++)
                            occ = any_hit(S.nodes, S.tris, root, pick3<NS>(sa, sg), pick3<NS>(sd, sg), 1.0f) < 1.0f;
                    }
                    if (occ) thr = 0.0f;
                } else if (nc > 0) {
                    // The nc x nv (candidate, root) tests are spread over all 32 lanes, candidate
                    // major (neighbouring lanes load the same triangle), instead of each root's lane
                    // testing every candidate while the lanes without a root idle.  A root is
                    // occluded when any of its tests hits before the segment's end; tests of roots
                    // already found occluded are skipped.
                    if (thr > 0.0f) {
#pragma unroll
                        for (int sg = 0; sg < NS; sg++) {
                            segA[warp][sg][0][lane] = sa[sg].x;
                            segA[warp][sg][1][lane] = sa[sg].y;
                            segA[warp][sg][2][lane] = sa[sg].z;
                            segD[warp][sg][0][lane] = sd[sg].x;
                            segD[warp][sg][1][lane] = sd[sg].y;
                            segD[warp][sg][2][lane] = sd[sg].z;
                        }
                    }
                    if (lane == 0) occMask[warp] = 0u;
                    __syncwarp();
                    const int nv = __popc(valid);
                    const int total = nc * nv;
                    const int dq = 32 / nv, dr = 32 % nv;
                    int c = lane / nv, rr = lane % nv;
                    volatile uint32_t* occ = &occMask[warp];
                    for (int pIdx = lane; pIdx < total; pIdx += 32) {
                        const int src = (int)__fns(valid, 0, rr + 1);
                        if (!((*occ >> src) & 1u)) {
                            const uint32_t e = cand[warp][c];
                            const uint32_t sg = e >> kSegShift;
                            float3 v0, v1, v2;
                            load_tri(S.tris, e & kIdxMask, v0, v1, v2);
                            float t, u, v;
                            float3 ng;
                            const float3 ro = mk3(segA[warp][sg][0][src], segA[warp][sg][1][src], segA[warp][sg][2][src]);
                            const float3 rd = mk3(segD[warp][sg][0][src], segD[warp][sg][1][src], segD[warp][sg][2][src]);
                            if (ray_triangle(&t, &u, &v, &ng, 0.0f, 1.0f, ro, rd, v0, v1, v2) &&
                                t < 1.0f)
                                atomicOr(&occMask[warp], 1u << src);
                        }
                        c += dq;
                        rr += dr;
                        if (rr >= nv) {
                            rr -= nv;
                            c++;
                        }
                    }
                    __syncwarp();
                    if ((occMask[warp] >> lane) & 1u) thr = 0.0f;
                }
                __syncwarp();
            }
            if (mine && !(thr > 0.0f)) acc[blk.first + idx].thr = 0.0f;
        }
        }
    }
    if (a.counters) {
        flush_count(a.counters + kCntQueries, cQueries);
        flush_count(a.counters + kCntFatOverflow, cOverflow);
        flush_count(a.counters + kCntCandidates, cCand);
    }
}

template <int K, bool kMulti>
__global__ void __launch_bounds__(256) k_p2_contrib(BatchArgs a)
{
    const int B = a.s.nBins;
    const unsigned long long n = min(a.p2[0], a.acceptCapacity);
    const auto* recs = reinterpret_cast<const PairRec<K>*>(a.records);
    const auto* acc = reinterpret_cast<const Accepted<K>*>(a.accepted);
    unsigned long long nContrib = 0;
    for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (unsigned long long)gridDim.x * blockDim.x) {
        const Accepted<K> e = acc[i];
        if (!(e.thr > 0.0f)) continue;
        const PairRec<K>& r = recs[e.rec];
        const SolveArgs& S = kMulti ? a.scenes[r.scene].s : a.s;
        const int4 ti = S.cache.tris[r.slot];
        const int tix[4] = {ti.x, ti.y, ti.z, ti.w};
        Chain<K> ch;
        load_chain<K>(ch, S.tris, S.attribs, tix);
        const FirstDiffuse fd = S.fds[r.pixel];
        const V3<float> p = v3f<float>(fd.p);
        const float eta = S.etas[e.bin];
        const float dadwv = dadw_out_of_line<K>(ch, e.x, S.p_light, fd.p, S.events, eta);
        const V3<float> vl = vertex<float, K>(ch, e.x, K - 1);
        const float cosv = fmaxf(vdot(vnormalize(vl - p), v3f<float>(fd.ng)), 0.0f);
        float contrib = e.thr * S.lightIntensity / dadwv * cosv;
        contrib = fminf(contrib, S.radianceClamp);
        atomicAdd(S.spectral + (size_t)r.pixel * B + e.bin, contrib);
        nContrib++;
    }
    if (a.s.stats) flush_count(a.s.stats + 2, nContrib);
}

template <int K, bool kMulti>
static cudaError_t launch_phases(const BatchArgs& a, int blocksPerSM, int p1BlocksPerSM, cudaStream_t s)
{
    const int sms = num_sms();
    k_probe<K, kMulti><<<sms * 2 * p1BlocksPerSM, 256, 0, s>>>(a);
    k_phase1<K, kMulti><<<sms * p1BlocksPerSM, 256, 0, s>>>(a);
    for (int w = 0; w < kMaxWaves; w++) {
        cudaError_t e = cudaMemsetAsync(a.p2, 0, 4 * sizeof(unsigned long long), s);
        if (e != cudaSuccess) return e;
        BatchArgs aw = a;
        aw.wave = w;
        k_p2_solve<K, kMulti><<<sms * blocksPerSM, kWarpsPerBlock * 32, 0, s>>>(aw);
        k_p2_vis<K, kMulti><<<sms * 3, kWarpsPerBlock * 32, 0, s>>>(aw);
        k_p2_contrib<K, kMulti><<<sms * 8, 256, 0, s>>>(aw);
    }
    return cudaGetLastError();
}

template <int K>
static cudaError_t launch_k(const BatchArgs& a, int blocksPerSM, cudaStream_t s, int p1BlocksPerSM = 8)
{
    if (a.scenes) return launch_phases<K, true>(a, blocksPerSM, p1BlocksPerSM, s);
    return launch_phases<K, false>(a, blocksPerSM, p1BlocksPerSM, s);
}

size_t probe_bytes(int K)
{
    switch (K) {
        case 1: return sizeof(Probe<1>);
        case 2: return sizeof(Probe<2>);
        case 3: return sizeof(Probe<3>);
        case 4: return sizeof(Probe<4>);
        default: return 0;
    }
}

size_t accepted_bytes(int K)
{
    switch (K) {
        case 1: return sizeof(Accepted<1>);
        case 2: return sizeof(Accepted<2>);
        case 3: return sizeof(Accepted<3>);
        case 4: return sizeof(Accepted<4>);
        default: return 0;
    }
}

size_t block_bytes() { return sizeof(AcceptBlock); }

size_t record_bytes(int K)
{
    switch (K) {
        case 1: return sizeof(PairRec<1>);
        case 2: return sizeof(PairRec<2>);
        case 3: return sizeof(PairRec<3>);
        case 4: return sizeof(PairRec<4>);
        default: return 0;
    }
}

cudaError_t launch_solve_batched(int K, const BatchArgs& a, int blocksPerSM, cudaStream_t s)
{
    if (a.s.nBins < 1 || a.s.nBins > 64) return cudaErrorInvalidValue;
    // work counter, record count and the second queue's two words are consecutive header words
    cudaError_t e = cudaMemsetAsync(a.workCounter, 0, 4 * sizeof(unsigned long long), s);
    if (e != cudaSuccess) return e;
    switch (K) {
        case 1: return launch_k<1>(a, blocksPerSM, s);
        case 2: return launch_k<2>(a, blocksPerSM, s);
        case 3: return launch_k<3>(a, blocksPerSM, s);
        case 4: return launch_k<4>(a, blocksPerSM, s);
    }
    return cudaErrorInvalidValue;
}

cudaError_t launch_solve_batched_multi(int K, const BatchArgs& a, int p1BlocksPerSM, int p2BlocksPerSM,
                                       unsigned long long* offsets, cudaStream_t s)
{
    if (a.s.nBins < 1 || a.s.nBins > 64 || !a.scenes || a.nScenes == 0) return cudaErrorInvalidValue;
    // work counter, record count and the second queue's two words are consecutive header words
    cudaError_t e = cudaMemsetAsync(a.workCounter, 0, 4 * sizeof(unsigned long long), s);
    if (e != cudaSuccess) return e;
    k_scene_offsets<<<1, 1024, 0, s>>>(a.scenes, a.nScenes, offsets);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    switch (K) {
        case 1: return launch_k<1>(a, p2BlocksPerSM, s, p1BlocksPerSM);
        case 2: return launch_k<2>(a, p2BlocksPerSM, s, p1BlocksPerSM);
        case 3: return launch_k<3>(a, p2BlocksPerSM, s, p1BlocksPerSM);
        case 4: return launch_k<4>(a, p2BlocksPerSM, s, p1BlocksPerSM);
    }
    return cudaErrorInvalidValue;
}

}  // namespace batched
}  // namespace pz
