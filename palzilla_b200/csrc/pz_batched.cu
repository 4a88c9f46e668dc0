// pz_batched.cu -- batched persistent specular solver (binned wavelengths).
//
// Same work items and results as the plain solver (one (pixel, tuple) work item solved
// for every wavelength bin, solveSpecularPath<K> semantics per bin), organised for the
// GPU:
//  * persistent warps pull chunks of 32 work items from a device counter (no host
//    round trip: the item count is read from device memory);
//  * phase 1, one lane per item: an unconstrained Newton solve at the centre bin from
//    the photon's barycentrics, and the derivative of the root with respect to eta from
//    the same Jacobian (implicit-function theorem).  The root of every other bin is
//    predicted linearly; bins whose predicted root lies outside the triangles by more
//    than kMargin are rejected without a solve, the rest are refined in phase 2.  Items
//    whose centre solve does not converge, or whose prediction is unreliable, fall back
//    to the plain per-bin solve from the photon's barycentrics;
//  * phase 2, one lane per bin: Newton with the reference's rules (multi-tangent duals:
//    one pass per iteration) from the photon's barycentrics, as the plain solver -- the
//    reference's accept/reject decision depends on the Newton path through its
//    shrinking edge test, so this keeps it -- or, with continuation enabled, from the
//    predicted root (fewer iterations, roots near triangle edges accepted more
//    often than the reference does); admissibility checks, then
//    visibility shared by the whole warp: for each path segment one BVH query with the
//    segment fattened to cover every bin's segment collects the few candidate
//    triangles, and each bin tests only those (exact: a triangle that cuts any bin's
//    segment lies within the fattening radius of the reference segment);
//  * FP64 polish: bins of items with |det R| < 1e-6 at the root (ill-conditioned) are
//    re-solved and re-checked in double precision from the FP32 root.
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
constexpr int kMaxCand = 32;
constexpr float kMaxShift = 0.5f;    // a larger predicted shift over the band falls back
constexpr float kDeep = 0.3f;        // a predicted root this far inside every triangle is refined, not re-solved

// Phase-1 result of one work item that has bins to refine (global, compacted).
template <int K> struct PairRec {
    int pixel, slot, mode;  // mode 1: predicted roots, 2: plain per-bin solves
    int polish;             // the item is ill-conditioned: FP64 polish of its roots
    unsigned long long mask;  // bins to solve (mode 1)
    unsigned long long warm;  // of those, bins whose root is deep inside: refine the prediction
    float xa[2 * K], xc[2 * K], xb[2 * K];  // roots at the first, centre and last bin
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

// The shadow-ray segment of occluded() (pk.h:88-115): start and end points.
PZ_D void shadow_segment(float3 from, float3 from_n, float3 to, float3 to_n, float3& a, float3& b)
{
    if (ex::dot(ex::sub3(to, from), from_n) < 0.0f) from_n = -from_n;
    if (ex::dot(ex::sub3(from, to), to_n) < 0.0f) to_n = -to_n;
    a = ex::add3(from, ex::mul3(from_n, ray_offset_scale(from)));
    b = ex::add3(to, ex::mul3(to_n, ray_offset_scale(to)));
}

// Warp-cooperative query: leaves whose box, grown by r, meets segment [a, b].  Every
// lane runs the same traversal; the candidate list goes to shared memory.  Returns the
// count, or -1 when the list overflows.
PZ_D int fat_query(const Node* __restrict__ nodes, const Tri* __restrict__ tris, uint32_t root, float3 a, float3 b,
                   float r, uint32_t* cand)
{
    const float3 d = b - a;
    const float3 inv = inv_rd(d);
    const float3 R = mk3(r, r, r);
    uint32_t stack[kStack];
    int sp = 0, n = 0;
    uint32_t node = root;
    while (node != kInvalidNode) {
        if (is_leaf(node)) {
            if (n < kMaxCand) {
                if ((threadIdx.x & 31) == 0) cand[n] = node_idx(node);
                n++;
            } else {
                return -1;
            }
            node = sp == 0 ? kInvalidNode : stack[--sp];
            continue;
        }
        const NodeView nv = load_node(nodes, node_idx(node));
        float rl, rr;
        const bool hl = slab_hit(a, inv, nv.lo0 - R, nv.hi0 + R, 1.0f, &rl);
        const bool hr = slab_hit(a, inv, nv.lo1 - R, nv.hi1 + R, 1.0f, &rr);
        if (hl && hr) {
            if (sp >= kStack) return -1;
            stack[sp++] = nv.c1;
            node = nv.c0;
        } else if (hl || hr) {
            node = hl ? nv.c0 : nv.c1;
        } else {
            node = sp == 0 ? kInvalidNode : stack[--sp];
        }
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

// ---------------------------------------------------------------- phase 1
template <int K>
__global__ void __launch_bounds__(256, 2) k_phase1(BatchArgs a)
{
    const int B = a.s.nBins;
    const uint64_t nPaths = a.nPathsDev ? min((uint64_t)*a.nPathsDev, a.s.nPaths) : a.s.nPaths;
    const int bc = B / 2;
    const float eta_c = a.s.etas[bc];
    const V3<float> L = v3f<float>(a.s.p_light);
    auto* recs = reinterpret_cast<PairRec<K>*>(a.records);
    unsigned long long nItems = 0;
    for (uint64_t idx = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < nPaths;
         idx += (uint64_t)gridDim.x * blockDim.x) {
        const SpecularPath sp = a.s.paths[idx];
        const int4 ti = a.s.cache.tris[sp.cacheIndex];
        const int tix[4] = {ti.x, ti.y, ti.z, ti.w};
        Chain<K> ch;
        load_chain<K>(ch, a.s.tris, a.s.attribs, tix);
        const float4 q0 = a.s.cache.params[2 * sp.cacheIndex], q1 = a.s.cache.params[2 * sp.cacheIndex + 1];
        const float pp[8] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
        float x[2 * K];
#pragma unroll
        for (int i = 0; i < 2 * K; i++) x[i] = pp[i];
        const V3<float> p = v3f<float>(a.s.fds[sp.pixel].p);
        int it;
        float det;
        const bool conv = newton<float, K>(x, L, p, ch, eta_c, a.s.events, 24, a.s.costTolerance, 0, false, &it, &det);
        PairRec<K> r;
        r.pixel = sp.pixel;
        r.slot = sp.cacheIndex;
        r.mode = 2;
        r.polish = 0;
        r.mask = 0;
        r.warm = 0;
        bool conv2 = false;
        if (conv && B >= 3) {
            // root derivative in eta at the centre (implicit-function theorem) and the two
            // end-bin roots, warm-started from the tangent prediction
            float J[2 * K + 1][3 * K], c[3 * K], cost;
            eval_constraints<float, K, true>(x, L, p, ch, eta_c, a.s.events, J, c, cost);
            float Jx[2 * K][3 * K], rhs[3 * K], dxe[2 * K];
#pragma unroll
            for (int i = 0; i < 2 * K; i++)
#pragma unroll
                for (int j = 0; j < 3 * K; j++) Jx[i][j] = J[i][j];
#pragma unroll
            for (int j = 0; j < 3 * K; j++) rhs[j] = J[2 * K][j];
            det = qr_solve_reldet<float, 3 * K, 2 * K>(Jx, rhs, dxe);
            const float ea = a.s.etas[0], eb = a.s.etas[B - 1];
            float lin_a[2 * K], lin_b[2 * K];
#pragma unroll
            for (int i = 0; i < 2 * K; i++) {
                r.xc[i] = x[i];
                lin_a[i] = x[i] - (ea - eta_c) * dxe[i];
                lin_b[i] = x[i] - (eb - eta_c) * dxe[i];
                r.xa[i] = lin_a[i];
                r.xb[i] = lin_b[i];
            }
            int ia, ib;
            float da, db;
            const bool ca =
                newton<float, K>(r.xa, L, p, ch, ea, a.s.events, 12, a.s.costTolerance, 0, false, &ia, &da, 1);
            const bool cb =
                newton<float, K>(r.xb, L, p, ch, eb, a.s.events, 12, a.s.costTolerance, 0, false, &ib, &db, 1);
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
            } else if (ca && cb && finite && nonlin < kMaxShift) {
                // A bin contributes only if its root lies inside every triangle, so a bin whose
                // predicted root is outside by more than the prediction error cannot contribute.
                const float err = 2.0f * nonlin + 1.0e-4f;
                unsigned long long mask = 0, warm = 0;
                for (int b = 0; b < B; b++) {
                    float xp[2 * K];
                    predict_root<K>(xp, r, a.s.etas[b], ea, eta_c, eb);
                    float depth = 1.0f;
#pragma unroll
                    for (int k = 0; k < K; k++)
                        depth = fminf(depth, fminf(fminf(xp[2 * k], xp[2 * k + 1]), 1.0f - xp[2 * k] - xp[2 * k + 1]));
                    if (depth > -err) mask |= 1ull << b;
                    if (depth > kDeep + err) warm |= 1ull << b;
                }
                r.mask = mask;
                r.warm = warm;
                r.mode = mask ? 1 : 0;
            }
        }
        nItems += (unsigned long long)B;
        if (a.counters) {
            atomicAdd(a.counters + r.mode, 1ull);
            if (r.mode == 2) atomicAdd(a.counters + (conv && conv2 ? kCntFallbackShift : kCntFallbackNoConv), 1ull);
        }
        // warp-aggregated append of the items that have work
        const bool keep = r.mode != 0;
        const uint32_t active = __activemask();
        const uint32_t ballot = __ballot_sync(active, keep);
        const int leader = __ffs(active) - 1;
        unsigned long long slot0 = 0;
        if ((int)(threadIdx.x & 31) == leader && ballot)
            slot0 = atomicAdd(a.recordCount, (unsigned long long)__popc(ballot));
        slot0 = __shfl_sync(active, slot0, leader);
        if (keep) {
            const unsigned long long dst = slot0 + __popc(ballot & ((1u << (threadIdx.x & 31)) - 1u));
            if (dst < a.recordCapacity) recs[dst] = r;
            else raise_error(a.status, kErrCapacity);
        }
    }
    if (a.s.stats) {
        const uint32_t active = __activemask();
        for (int o = 16; o > 0; o >>= 1) nItems += __shfl_xor_sync(active, nItems, o);
        if ((threadIdx.x & 31) == 0) atomicAdd(a.s.stats + 0, nItems);
    }
}

// ---------------------------------------------------------------- phase 2
template <int K>
__global__ void __launch_bounds__(kWarpsPerBlock * 32, 2) k_phase2(BatchArgs a)
{
    __shared__ uint32_t cand[kWarpsPerBlock][kMaxCand];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int B = a.s.nBins;
    const unsigned long long nRec = min(*a.recordCount, a.recordCapacity);
    const auto* recs = reinterpret_cast<const PairRec<K>*>(a.records);
    const uint32_t root = __ldg(a.s.root);
    const float eta_c = a.s.etas[B / 2];
    const V3<float> L = v3f<float>(a.s.p_light);
    unsigned long long nConv = 0, nContrib = 0;
    for (;;) {
        unsigned long long j = 0;
        if (lane == 0) j = atomicAdd(a.workCounter, 1ull);
        j = __shfl_sync(0xFFFFFFFFu, j, 0);
        if (j >= nRec) break;
        const PairRec<K> r = recs[j];
        const int4 ti = a.s.cache.tris[r.slot];
        const int tix[4] = {ti.x, ti.y, ti.z, ti.w};
        Chain<K> ch;
        load_chain<K>(ch, a.s.tris, a.s.attribs, tix);
        const FirstDiffuse fd = a.s.fds[r.pixel];
        const V3<float> p = v3f<float>(fd.p);
        float x0[2 * K];
        {
            const float4 q0 = a.s.cache.params[2 * r.slot], q1 = a.s.cache.params[2 * r.slot + 1];
            const float pp[8] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
#pragma unroll
            for (int i = 0; i < 2 * K; i++) x0[i] = pp[i];
        }
        // lanes take the bins to solve in rank order (the set bits of the item's mask)
        const unsigned long long todo = r.mode == 2 ? (B == 64 ? ~0ull : ((1ull << B) - 1ull)) : r.mask;
#if PZ_BATCHED_RANK
        const int nTodo = __popcll(todo);
        for (int round = 0; round * 32 < nTodo; round++) {
            const int rank = lane + 32 * round;
            const int b = rank < nTodo ? nth_bit64(todo, rank) : B;
#else
        for (int round = 0; round * 32 < B; round++) {
            const int b0 = lane + 32 * round;
            const int b = (b0 < B && ((todo >> b0) & 1ull)) ? b0 : B;
#endif
            float xs[2 * K];
            float thr = 0.0f;
            if (b < B) {
                const float eta = a.s.etas[b];
                const bool warm = r.mode == 1 && (a.continuation || ((r.warm >> b) & 1ull));
                if (warm) {
                    predict_root<K>(xs, r, eta, a.s.etas[0], eta_c, a.s.etas[B - 1]);
                } else {
#pragma unroll
                    for (int i = 0; i < 2 * K; i++) xs[i] = x0[i];
                }
                int it;
                float det;
                const bool conv = newton<float, K>(xs, L, p, ch, eta, a.s.events, a.s.maxIterations,
                                                   a.s.costTolerance, a.s.earlyTermWarmUp, true, &it, &det,
                                                   warm ? 1 : 0);
                if (a.counters) atomicAdd(a.counters + kCntNewton2, 1ull);
                if (conv) {
                    nConv++;
                    const bool polish = r.polish || (double)det < a.polishDet;
                    if (polish && a.counters) atomicAdd(a.counters + kCntPolish, 1ull);
                    float3 vtx[K + 2], nrm[K + 2];
                    if (polish)
                        thr = polish_fp64<K>(xs, ch, a.s.p_light, fd.p, a.s.events, eta, vtx, nrm);
                    else
                        thr = pre_throughput<float, K>(xs, L, p, ch, a.s.events, eta, vtx, nrm);
                }
            }
            // shared visibility: one fattened query per segment for all bins of the round
            for (int s = 0; s < K + 1; s++) {
                const uint32_t valid = __ballot_sync(0xFFFFFFFFu, thr > 0.0f);
                if (!valid) break;
                const int leader = __ffs(valid) - 1;
                float3 sa = mk3(0.f, 0.f, 0.f), sb = mk3(0.f, 0.f, 0.f);
                if (thr > 0.0f) {
                    float3 v0, n0, v1, n1;
                    chain_vertex<K>(ch, xs, a.s.p_light, fd.p, s, v0, n0);
                    chain_vertex<K>(ch, xs, a.s.p_light, fd.p, s + 1, v1, n1);
                    shadow_segment(v0, n0, v1, n1, sa, sb);
                }
                const float3 ra = mk3(__shfl_sync(0xFFFFFFFFu, sa.x, leader), __shfl_sync(0xFFFFFFFFu, sa.y, leader),
                                      __shfl_sync(0xFFFFFFFFu, sa.z, leader));
                const float3 rb = mk3(__shfl_sync(0xFFFFFFFFu, sb.x, leader), __shfl_sync(0xFFFFFFFFu, sb.y, leader),
                                      __shfl_sync(0xFFFFFFFFu, sb.z, leader));
                float rad = 0.0f, mag = 0.0f;
                if (thr > 0.0f) {
                    const float3 da = vabs(sa - ra), db = vabs(sb - rb);
                    rad = fmaxf(fmaxf(fmaxf(da.x, da.y), da.z), fmaxf(fmaxf(db.x, db.y), db.z));
                    const float3 ma = vabs(sa), mb = vabs(sb);
                    mag = fmaxf(fmaxf(fmaxf(ma.x, ma.y), ma.z), fmaxf(fmaxf(mb.x, mb.y), mb.z));
                }
                rad = warp_max(rad);
                mag = warp_max(mag);
                rad += 1.0e-5f * (1.0f + mag);  // covers the rounding of the slab and box arithmetic
                const int nc = fat_query(a.s.nodes, a.s.tris, root, ra, rb, rad, cand[warp]);
                __syncwarp();
                if (lane == 0 && a.counters) {
                    atomicAdd(a.counters + kCntQueries, 1ull);
                    if (nc < 0) atomicAdd(a.counters + kCntFatOverflow, 1ull);
                    else atomicAdd(a.counters + kCntCandidates, (unsigned long long)nc);
                }
                if (thr > 0.0f) {
                    const float3 d = ex::sub3(sb, sa);
                    bool occ = false;
                    if (nc < 0) {
                        occ = any_hit(a.s.nodes, a.s.tris, root, sa, d, 1.0f) < 1.0f;
                    } else {
                        for (int c = 0; c < nc && !occ; c++) {
                            float3 v0, v1, v2;
                            load_tri(a.s.tris, cand[warp][c], v0, v1, v2);
                            float t, u, v;
                            float3 ng;
                            if (ray_triangle(&t, &u, &v, &ng, 0.0f, 1.0f, sa, d, v0, v1, v2) && t < 1.0f) occ = true;
                        }
                    }
                    if (occ) thr = 0.0f;
                }
                __syncwarp();
            }
            if (thr > 0.0f) {
                nContrib++;
                const float eta = a.s.etas[b];
                const float dadwv = dadw_out_of_line<K>(ch, xs, a.s.p_light, fd.p, a.s.events, eta);
                const V3<float> vl = vertex<float, K>(ch, xs, K - 1);
                const float cosv = fmaxf(vdot(vnormalize(vl - p), v3f<float>(fd.ng)), 0.0f);
                float contrib = thr * a.s.lightIntensity / dadwv * cosv;
                contrib = fminf(contrib, a.s.radianceClamp);
                atomicAdd(a.s.spectral + (size_t)r.pixel * B + b, contrib);
            }
        }
    }
    if (a.s.stats) {
        for (int o = 16; o > 0; o >>= 1) {
            nConv += __shfl_xor_sync(0xFFFFFFFFu, nConv, o);
            nContrib += __shfl_xor_sync(0xFFFFFFFFu, nContrib, o);
        }
        if (lane == 0) {
            atomicAdd(a.s.stats + 1, nConv);
            atomicAdd(a.s.stats + 2, nContrib);
        }
    }
}

template <int K>
static cudaError_t launch_k(const BatchArgs& a, int blocksPerSM, cudaStream_t s)
{
    k_phase1<K><<<kNumSMs * 8, 256, 0, s>>>(a);
    k_phase2<K><<<kNumSMs * blocksPerSM, kWarpsPerBlock * 32, 0, s>>>(a);
    return cudaGetLastError();
}

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
    cudaError_t e = cudaMemsetAsync(a.workCounter, 0, sizeof(unsigned long long), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(a.recordCount, 0, sizeof(unsigned long long), s);
    if (e != cudaSuccess) return e;
    switch (K) {
        case 1: return launch_k<1>(a, blocksPerSM, s);
        case 2: return launch_k<2>(a, blocksPerSM, s);
        case 3: return launch_k<3>(a, blocksPerSM, s);
        case 4: return launch_k<4>(a, blocksPerSM, s);
    }
    return cudaErrorInvalidValue;
}

}  // namespace batched
}  // namespace pz
