// pz_pathcuts.cu -- Path Cuts on the GPU: enumeration of the admissible K-triangle tuples
// of a specular chain between two points by interval culling over BVH node tuples
// (traverseAdmissibleNodes<K>, pk.h:1760-2220; normal bounds main.cpp:250-295).
//
// The reference walks the node-tuple tree depth first, one query at a time, on the CPU.
// Here every query's frontier of node tuples is expanded level by level: one thread per
// frontier entry picks the node to cut (largest surface area, the reference's rule and
// tie-break), tests both children with interval arithmetic and appends the admissible
// ones to the next frontier (warp-aggregated atomics); all-leaf tuples pass the
// reference's facing checks and go to the output list.  The set of tuples does not
// depend on the traversal order, only on the cut sequence of each branch, which is the
// reference's; the output order is not the reference's callback order.
//
// Arithmetic: round-to-nearest in the reference's operation order (this unit is built
// with -fmad=false), which reproduces the reference's tuple set exactly, or directed
// rounding (every bound rounded outward), which makes the culling conservative: its
// tuple set contains the round-to-nearest one.
#include <algorithm>

#include "pz_capi_internal.h"
#include "pz_common.cuh"

namespace pz {
namespace cuts {

constexpr int kBlock = 256;
constexpr int kMaxK = 4;

// ---------------------------------------------------------------- rounding policies
struct RN {
    static PZ_D float add_d(float a, float b) { return __fadd_rn(a, b); }
    static PZ_D float add_u(float a, float b) { return __fadd_rn(a, b); }
    static PZ_D float sub_d(float a, float b) { return __fsub_rn(a, b); }
    static PZ_D float sub_u(float a, float b) { return __fsub_rn(a, b); }
    static PZ_D float mul_d(float a, float b) { return __fmul_rn(a, b); }
    static PZ_D float mul_u(float a, float b) { return __fmul_rn(a, b); }
    static PZ_D float div_d(float a, float b) { return __fdiv_rn(a, b); }
    static PZ_D float div_u(float a, float b) { return __fdiv_rn(a, b); }
    static PZ_D float sqrt_d(float a) { return __fsqrt_rn(a); }
    static PZ_D float sqrt_u(float a) { return __fsqrt_rn(a); }
};
struct DR {
    static PZ_D float add_d(float a, float b) { return __fadd_rd(a, b); }
    static PZ_D float add_u(float a, float b) { return __fadd_ru(a, b); }
    static PZ_D float sub_d(float a, float b) { return __fsub_rd(a, b); }
    static PZ_D float sub_u(float a, float b) { return __fsub_ru(a, b); }
    static PZ_D float mul_d(float a, float b) { return __fmul_rd(a, b); }
    static PZ_D float mul_u(float a, float b) { return __fmul_ru(a, b); }
    static PZ_D float div_d(float a, float b) { return __fdiv_rd(a, b); }
    static PZ_D float div_u(float a, float b) { return __fdiv_ru(a, b); }
    static PZ_D float sqrt_d(float a) { return __fsqrt_rd(a); }
    static PZ_D float sqrt_u(float a) { return __fsqrt_ru(a); }
};

PZ_D float smin(float a, float b) { return a < b ? a : b; }
PZ_D float smax(float a, float b) { return a > b ? a : b; }

// ---------------------------------------------------------------- intervals (interval.h:34-713)
struct Iv { float l, u; };
struct Iv3 { Iv x, y, z; };

PZ_D Iv ival(float v) { return Iv{v, v}; }
PZ_D Iv ineg(Iv a) { return Iv{-a.u, -a.l}; }
template <class P> PZ_D Iv iadd(Iv a, Iv b) { return Iv{P::add_d(a.l, b.l), P::add_u(a.u, b.u)}; }
template <class P> PZ_D Iv isub(Iv a, Iv b) { return Iv{P::sub_d(a.l, b.u), P::sub_u(a.u, b.l)}; }
template <class P> PZ_D Iv imul(Iv a, Iv b)
{
    const float d0 = P::mul_d(a.l, b.l), d1 = P::mul_d(a.l, b.u), d2 = P::mul_d(a.u, b.l), d3 = P::mul_d(a.u, b.u);
    const float u0 = P::mul_u(a.l, b.l), u1 = P::mul_u(a.l, b.u), u2 = P::mul_u(a.u, b.l), u3 = P::mul_u(a.u, b.u);
    return Iv{smin(d0, smin(d1, smin(d2, d3))), smax(u0, smax(u1, smax(u2, u3)))};
}
template <class P> PZ_D Iv isqrt(Iv a) { return Iv{P::sqrt_d(a.l), P::sqrt_u(a.u)}; }
template <class P> PZ_D Iv isquare(Iv a)
{
    const float larger = smax(P::mul_u(a.l, a.l), P::mul_u(a.u, a.u));
    if (a.l <= 0.0f && 0.0f <= a.u) return Iv{0.0f, larger};
    return Iv{smin(P::mul_d(a.l, a.l), P::mul_d(a.u, a.u)), larger};
}

PZ_D Iv3 i3(float3 v) { return Iv3{ival(v.x), ival(v.y), ival(v.z)}; }
PZ_D Iv3 i3(const Box& b) { return Iv3{{b.lo.x, b.hi.x}, {b.lo.y, b.hi.y}, {b.lo.z, b.hi.z}}; }
PZ_D Iv3 ineg3(Iv3 a) { return Iv3{ineg(a.x), ineg(a.y), ineg(a.z)}; }
template <class P> PZ_D Iv3 iadd3(Iv3 a, Iv3 b) { return Iv3{iadd<P>(a.x, b.x), iadd<P>(a.y, b.y), iadd<P>(a.z, b.z)}; }
template <class P> PZ_D Iv3 isub3(Iv3 a, Iv3 b) { return Iv3{isub<P>(a.x, b.x), isub<P>(a.y, b.y), isub<P>(a.z, b.z)}; }
template <class P> PZ_D Iv3 imul3(Iv3 a, Iv s) { return Iv3{imul<P>(a.x, s), imul<P>(a.y, s), imul<P>(a.z, s)}; }
template <class P> PZ_D Iv idot(Iv3 a, Iv3 b)
{
    return iadd<P>(iadd<P>(imul<P>(a.x, b.x), imul<P>(a.y, b.y)), imul<P>(a.z, b.z));
}
template <class P> PZ_D Iv3 icross(Iv3 a, Iv3 b)
{
    return Iv3{isub<P>(imul<P>(a.y, b.z), imul<P>(a.z, b.y)), isub<P>(imul<P>(a.z, b.x), imul<P>(a.x, b.z)),
               isub<P>(imul<P>(a.x, b.y), imul<P>(a.y, b.x))};
}
template <class P> PZ_D Iv ilength_sq(Iv3 v)
{
    return iadd<P>(iadd<P>(isquare<P>(v.x), isquare<P>(v.y)), isquare<P>(v.z));
}
// l * u <= 0 on every axis; with directed rounding the product rounds toward -inf, so a
// test that round-to-nearest passes passes here too.
template <class P> PZ_D bool zero_included(Iv3 v)
{
    return P::mul_d(v.x.l, v.x.u) <= 0.0f && P::mul_d(v.y.l, v.y.u) <= 0.0f && P::mul_d(v.z.l, v.z.u) <= 0.0f;
}

// interval.h:229-252
template <class P> PZ_D Iv3 ireflection(Iv3 wi, Iv3 n)
{
    const float eps = 1.0e-10f;
    const Iv nxx = isquare<P>(n.x), nyy = isquare<P>(n.y), nzz = isquare<P>(n.z);
    const Iv nn = iadd<P>(iadd<P>(nxx, nyy), nzz);
    const Iv s{P::div_d(2.0f, smax(nn.u, eps)), P::div_u(2.0f, smax(nn.l, eps))};
    const Iv one = ival(1.0f);
    const Iv m11 = isub<P>(imul<P>(s, nxx), one), m12 = imul<P>(imul<P>(s, n.x), n.y),
             m13 = imul<P>(imul<P>(s, n.x), n.z);
    const Iv m21 = m12, m22 = isub<P>(imul<P>(s, nyy), one), m23 = imul<P>(imul<P>(s, n.y), n.z);
    const Iv m31 = m13, m32 = m23, m33 = isub<P>(imul<P>(s, nzz), one);
    return Iv3{iadd<P>(iadd<P>(imul<P>(m11, wi.x), imul<P>(m12, wi.y)), imul<P>(m13, wi.z)),
               iadd<P>(iadd<P>(imul<P>(m21, wi.x), imul<P>(m22, wi.y)), imul<P>(m23, wi.z)),
               iadd<P>(iadd<P>(imul<P>(m31, wi.x), imul<P>(m32, wi.y)), imul<P>(m33, wi.z))};
}

// interval.h:254-259
template <class P> PZ_D Iv3 irefraction_normal(Iv3 wi, Iv3 wo, Iv eta)
{
    const Iv lenWi = isqrt<P>(ilength_sq<P>(wi));
    const Iv lenWo = isqrt<P>(ilength_sq<P>(wo));
    return ineg3(iadd3<P>(imul3<P>(imul3<P>(wo, lenWi), eta), imul3<P>(wi, lenWo)));
}

// interval.h:398-418; em1 = eta * eta - 1
template <class P> PZ_D bool irefraction_norm_free(Iv3* wo, Iv3 wi, Iv3 n, Iv em1)
{
    const Iv NoN = ilength_sq<P>(n);
    Iv WIoN = idot<P>(wi, n);
    if (WIoN.u < 0.0f) return false;
    WIoN.l = smax(WIoN.l, 0.0f);
    const Iv WIoWI = ilength_sq<P>(wi);
    Iv k = iadd<P>(imul<P>(imul<P>(NoN, WIoWI), em1), isquare<P>(WIoN));
    if (k.u < 0.0f) return false;
    k.l = smax(k.l, 0.0f);
    *wo = iadd3<P>(imul3<P>(ineg3(wi), NoN), imul3<P>(n, isub<P>(WIoN, isqrt<P>(k))));
    return true;
}

// x / sqrt(q) with q in [ql, qu] (q >= eps^2 clamp applied to the root), rounded outward:
// the lower bound takes the root that moves x toward -inf, the upper the other one.
template <class P> PZ_D float ndiv_d(float x, float lenLo, float lenHi)
{
    return 0.0f <= x ? P::div_d(x, lenHi) : P::div_d(x, lenLo);
}
template <class P> PZ_D float ndiv_u(float x, float lenLo, float lenHi)
{
    return 0.0f <= x ? P::div_u(x, lenLo) : P::div_u(x, lenHi);
}

// interval.h:479-679 (the branch the reference compiles)
template <class P> PZ_D Iv3 inormalize(Iv3 p)
{
    const float eps = 1.0e-10f;
    if (P::mul_d(p.x.l, p.x.u) <= 0.0f && P::mul_d(p.y.l, p.y.u) <= 0.0f && P::mul_d(p.z.l, p.z.u) <= 0.0f)
        return Iv3{{-1.0f, 1.0f}, {-1.0f, 1.0f}, {-1.0f, 1.0f}};
    const float vs[3][2] = {{p.x.l, p.x.u}, {p.y.l, p.y.u}, {p.z.l, p.z.u}};
    float bd[3][2] = {{2.0f, -2.0f}, {2.0f, -2.0f}, {2.0f, -2.0f}};
#pragma unroll
    for (int iz = 0; iz < 2; iz++)
#pragma unroll
        for (int iy = 0; iy < 2; iy++)
#pragma unroll
            for (int ix = 0; ix < 2; ix++) {
                const float x = vs[0][ix], y = vs[1][iy], z = vs[2][iz];
                const float lenLo = smax(
                    P::sqrt_d(P::add_d(P::add_d(P::mul_d(x, x), P::mul_d(y, y)), P::mul_d(z, z))), eps);
                const float lenHi = smax(
                    P::sqrt_u(P::add_u(P::add_u(P::mul_u(x, x), P::mul_u(y, y)), P::mul_u(z, z))), eps);
                const float c[3] = {x, y, z};
#pragma unroll
                for (int a = 0; a < 3; a++) {
                    bd[a][0] = smin(bd[a][0], ndiv_d<P>(c[a], lenLo, lenHi));
                    bd[a][1] = smax(bd[a][1], ndiv_u<P>(c[a], lenLo, lenHi));
                }
            }
    if (0.0f < vs[0][0] * vs[0][1] && 0.0f < vs[1][0] * vs[1][1] && 0.0f < vs[2][0] * vs[2][1])
        return Iv3{{bd[0][0], bd[0][1]}, {bd[1][0], bd[1][1]}, {bd[2][0], bd[2][1]}};
#pragma unroll
    for (int axis = 0; axis < 3; axis++) {
        const int ab = (axis + 1) % 3, ac = (axis + 2) % 3;
        if (0.0f < vs[axis][0] * vs[axis][1]) {
            const float nz = 0.0f < vs[axis][0] ? vs[axis][0] : vs[axis][1];
            const float nzzD = P::mul_d(nz, nz), nzzU = P::mul_u(nz, nz);
            const bool zx = vs[ab][0] * vs[ab][1] <= 0.0f;
            const bool zy = vs[ac][0] * vs[ac][1] <= 0.0f;
            if (zy) {
                const float lo = vs[ab][0], up = vs[ab][1];
                const float llLo = smax(P::sqrt_d(P::add_d(nzzD, P::mul_d(lo, lo))), eps);
                const float llHi = smax(P::sqrt_u(P::add_u(nzzU, P::mul_u(lo, lo))), eps);
                const float ulLo = smax(P::sqrt_d(P::add_d(nzzD, P::mul_d(up, up))), eps);
                const float ulHi = smax(P::sqrt_u(P::add_u(nzzU, P::mul_u(up, up))), eps);
                bd[ab][0] = smin(bd[ab][0], ndiv_d<P>(lo, llLo, llHi));
                bd[ab][1] = smax(bd[ab][1], ndiv_u<P>(up, ulLo, ulHi));
            }
            if (zx) {
                const float lo = vs[ac][0], up = vs[ac][1];
                const float llLo = smax(P::sqrt_d(P::add_d(nzzD, P::mul_d(lo, lo))), eps);
                const float llHi = smax(P::sqrt_u(P::add_u(nzzU, P::mul_u(lo, lo))), eps);
                const float ulLo = smax(P::sqrt_d(P::add_d(nzzD, P::mul_d(up, up))), eps);
                const float ulHi = smax(P::sqrt_u(P::add_u(nzzU, P::mul_u(up, up))), eps);
                bd[ac][0] = smin(bd[ac][0], ndiv_d<P>(lo, llLo, llHi));
                bd[ac][1] = smax(bd[ac][1], ndiv_u<P>(up, ulLo, ulHi));
            }
            if (zx && zy) {
                if (0.0f <= vs[axis][1]) bd[axis][1] = 1.0f;
                else bd[axis][0] = -1.0f;
            }
        }
    }
    return Iv3{{bd[0][0], bd[0][1]}, {bd[1][0], bd[1][1]}, {bd[2][0], bd[2][1]}};
}

// ---------------------------------------------------------------- BVH helpers
struct NormalBound { Box bounds[2]; uint32_t counter; };  // InternalNormalBound, pk.h:1705-1709
static_assert(sizeof(NormalBound) == 52, "InternalNormalBound layout");

PZ_D Box node_box(const Node& n)  // nodeAABB: the union of the two child boxes
{
    Box b = n.boxes[0];
    box_extend(b, n.boxes[1]);
    return b;
}
PZ_D float surface_area(const Box& b)  // minimum_lbvh.h:256-260
{
    const float3 s = b.hi - b.lo;
    return (s.x * s.y + s.y * s.z + s.z * s.x) * 2.0f;
}
PZ_D Box tri_box(const Tri& t)
{
    Box b = box_empty();
    box_extend(b, t.v0);
    box_extend(b, t.v1);
    box_extend(b, t.v2);
    return b;
}
PZ_D Box normal_box(const Attrib& a)
{
    Box b = box_empty();
    box_extend(b, a.n0);
    box_extend(b, a.n1);
    box_extend(b, a.n2);
    return b;
}

struct CutArgs {
    int K;
    uint32_t events;
    float eta;
    float3 pBeg;
    const float3* pEnd;        // one receiver point per query
    uint32_t nQueries;
    const Node* nodes;
    const NormalBound* nbs;
    const Tri* tris;
    const Attrib* attribs;
    const uint32_t* root;
    const uint32_t* frontIn;   // (1 + K) u32 per entry: query, node[K]
    const unsigned long long* countIn;
    uint32_t* frontOut;
    unsigned long long* countOut;
    uint32_t frontCapacity;
    uint32_t* tuples;          // (1 + K) u32 per tuple: query, triangle[K]
    unsigned long long* nTuples;
    uint32_t tupleCapacity;
    uint32_t* status;
};

// warp-aggregated append: each lane with `want` gets its own slot from *counter
PZ_D unsigned long long warp_append(unsigned long long* counter, bool want)
{
    const uint32_t active = __activemask();
    const uint32_t ballot = __ballot_sync(active, want);
    const int leader = __ffs(active) - 1;
    unsigned long long base = 0;
    if ((int)(threadIdx.x & 31) == leader && ballot) base = atomicAdd(counter, (unsigned long long)__popc(ballot));
    base = __shfl_sync(active, base, leader);
    return base + __popc(ballot & ((1u << (threadIdx.x & 31)) - 1u));
}

__global__ void k_cuts_init(CutArgs a)
{
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= a.nQueries) return;
    const uint32_t root = *a.root;
    uint32_t* e = a.frontOut + (size_t)q * (1 + a.K);
    e[0] = q;
    for (int k = 0; k < a.K; k++) e[1 + k] = root;
    if (q == 0) *a.countOut = a.nQueries;
}

template <int K, class P>
__global__ void __launch_bounds__(kBlock) k_cuts_round(CutArgs a)
{
    const uint32_t nIn = (uint32_t)min(*a.countIn, (unsigned long long)a.frontCapacity);
    const Iv etaIv = ival(a.eta);
    const Iv etaInv{P::div_d(1.0f, a.eta), P::div_u(1.0f, a.eta)};
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < nIn; e += gridDim.x * blockDim.x) {
        const uint32_t* ent = a.frontIn + (size_t)e * (1 + K);
        const uint32_t q = ent[0];
        uint32_t cur[K];
        bool empty = false;
#pragma unroll
        for (int k = 0; k < K; k++) {
            cur[k] = ent[1 + k];
            empty = empty || cur[k] == kInvalidNode;  // a BVH of no triangles
        }
        if (empty) continue;
        const float3 pEnd = a.pEnd[q];
        int cut = -1;
        float maxSA = -1.0f;
#pragma unroll
        for (int k = 0; k < K; k++) {
            if (is_leaf(cur[k])) continue;
            const float sa = surface_area(node_box(a.nodes[node_idx(cur[k])]));
            if (maxSA < sa) {
                cut = k;
                maxSA = sa;
            }
        }
        bool emit = false, push[2] = {false, false};
        uint32_t child[2] = {0u, 0u};
        if (cut == -1) {
            // every node is a triangle: the reference's checks before its callback
            bool invalid = false;
#pragma unroll
            for (int k = 0; k + 1 < K; k++)
                if (node_idx(cur[k]) == node_idx(cur[k + 1])) invalid = true;
            {
                const Tri tb = a.tris[node_idx(cur[0])];
                float3 ng = cross(tb.v1 - tb.v0, tb.v2 - tb.v0);
                ng = ng * dot(ng, a.attribs[node_idx(cur[0])].n0);
                if (dot(ng, a.pBeg) < dot(ng, tb.v0)) invalid = true;
            }
            {
                const Tri te = a.tris[node_idx(cur[K - 1])];
                float3 ng = cross(te.v1 - te.v0, te.v2 - te.v0);
                ng = ng * dot(ng, a.attribs[node_idx(cur[K - 1])].n0);
                if (dot(ng, pEnd) < dot(ng, te.v0)) invalid = true;
            }
            emit = !invalid;
        } else {
            const Node& cn = a.nodes[node_idx(cur[cut])];
#pragma unroll
            for (int i = 0; i < 2; i++) {
                Iv3 vtx[K + 2], nrm[K];
                vtx[0] = i3(a.pBeg);
                vtx[K + 1] = i3(pEnd);
#pragma unroll
                for (int k = 0; k < K; k++) {
                    const uint32_t nd = cur[k];
                    if (k == cut) {
                        vtx[k + 1] = i3(cn.boxes[i]);
                        nrm[k] = i3(a.nbs[node_idx(nd)].bounds[i]);
                    } else if (is_leaf(nd)) {
                        vtx[k + 1] = i3(tri_box(a.tris[node_idx(nd)]));
                        nrm[k] = i3(normal_box(a.attribs[node_idx(nd)]));
                    } else {
                        vtx[k + 1] = i3(node_box(a.nodes[node_idx(nd)]));
                        Box nb = box_empty();
                        box_extend(nb, a.nbs[node_idx(nd)].bounds[0]);
                        box_extend(nb, a.nbs[node_idx(nd)].bounds[1]);
                        nrm[k] = i3(nb);
                    }
                }
                bool admissible = true, inMedium = false;
                Iv3 wi = isub3<P>(vtx[0], vtx[1]);
#pragma unroll
                for (int k = 0; k < K; k++) {
                    if (!admissible) break;
                    const Iv3 wo = isub3<P>(vtx[k + 2], vtx[k + 1]);
                    Iv3 woNext;
                    if (!((a.events >> k) & 1u)) {
                        woNext = ireflection<P>(wi, nrm[k]);
                    } else {
                        const Iv e = inMedium ? etaInv : etaIv;
                        const Iv em1 = isub<P>(imul<P>(e, e), ival(1.0f));
                        const Iv3 wiv = isub3<P>(vtx[k], vtx[k + 1]);
                        const Iv3 ht = irefraction_normal<P>(wiv, wo, e);
                        if (!zero_included<P>(icross<P>(nrm[k], ht))) {
                            admissible = false;
                            break;
                        }
                        if (!irefraction_norm_free<P>(&woNext, wi, inMedium ? ineg3(nrm[k]) : nrm[k], em1)) {
                            admissible = false;
                            break;
                        }
                    }
                    if (!zero_included<P>(icross<P>(woNext, wo))) {
                        admissible = false;
                        break;
                    }
                    inMedium = !inMedium;
                    wi = ineg3(woNext);
                }
                push[i] = admissible;
                child[i] = cn.children[i];
            }
        }
        // leaf tuples to the output list
        {
            const unsigned long long slot = warp_append(a.nTuples, emit);
            if (emit) {
                if (slot < a.tupleCapacity) {
                    uint32_t* o = a.tuples + slot * (1 + K);
                    o[0] = q;
#pragma unroll
                    for (int k = 0; k < K; k++) o[1 + k] = node_idx(cur[k]);
                } else {
                    raise_error(a.status, kErrCapacity);
                }
            }
        }
        // admissible children to the next frontier
#pragma unroll
        for (int i = 0; i < 2; i++) {
            const unsigned long long slot =
                warp_append(a.countOut, push[i]);
            if (push[i]) {
                if (slot < a.frontCapacity) {
                    uint32_t* o = a.frontOut + slot * (1 + K);
                    o[0] = q;
#pragma unroll
                    for (int k = 0; k < K; k++) o[1 + k] = k == cut ? child[i] : cur[k];
                } else {
                    raise_error(a.status, kErrCapacity);
                }
            }
        }
    }
}

// Normal bounds of every internal node's two children (main.cpp:250-295): from each
// leaf upward, the second arriving child merges its sibling's bound and goes on.
__global__ void k_normal_bounds(const Node* __restrict__ nodes, uint32_t nInternals, const Attrib* __restrict__ attribs,
                                NormalBound* nbs)
{
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 2 * nInternals) return;
    const uint32_t i = t >> 1, j = t & 1;
    uint32_t me = nodes[i].children[j];
    if (!is_leaf(me)) return;
    Box nb = normal_box(attribs[node_idx(me)]);
    uint32_t parent = make_node(i, false);
    for (uint32_t depth = 0; parent != kInvalidNode && depth < 0x7FFFFFFFu; depth++) {
        NormalBound* pb = nbs + node_idx(parent);
        const int ci = nodes[node_idx(parent)].children[0] == me ? 0 : 1;
        volatile float* dst = reinterpret_cast<volatile float*>(&pb->bounds[ci]);
        dst[0] = nb.lo.x; dst[1] = nb.lo.y; dst[2] = nb.lo.z;
        dst[3] = nb.hi.x; dst[4] = nb.hi.y; dst[5] = nb.hi.z;
        __threadfence();
        const uint32_t v = atomicAdd(&pb->counter, 1u);
        if (v == 0) break;
        __threadfence();
        const volatile float* src = reinterpret_cast<const volatile float*>(&pb->bounds[ci ^ 1]);
        const Box sib{mk3(src[0], src[1], src[2]), mk3(src[3], src[4], src[5])};
        box_extend(nb, sib);
        me = parent;
        parent = nodes[node_idx(me)].parent;
    }
}

}  // namespace cuts
}  // namespace pz

using namespace pz;
using namespace pz::cuts;

static_assert(sizeof(pz_normal_bound) == sizeof(NormalBound), "pz_normal_bound layout");

namespace {
constexpr size_t kHeader = 256;  // status | count[2] | tuple count
size_t entry_bytes(int K) { return (size_t)(1 + K) * sizeof(uint32_t); }
}  // namespace

extern "C" int pz_normal_bounds(const pz_internal_node* internals_dev, int n_internals,
                                const pz_triangle_attrib* attribs_dev, pz_normal_bound* out_dev, pz_stream_t stream)
{
    if (n_internals < 0 || (n_internals > 0 && (!internals_dev || !attribs_dev || !out_dev)))
        return fail(PZ_ERR_INVALID_ARGUMENT, "pz_normal_bounds: bad argument");
    if (n_internals == 0) { clear_error(); return PZ_OK; }
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(out_dev, 0, sizeof(NormalBound) * (size_t)n_internals, s);
    if (e == cudaSuccess) {
        const uint32_t threads = 2u * (uint32_t)n_internals;
        k_normal_bounds<<<(threads + kBlock - 1) / kBlock, kBlock, 0, s>>>(
            reinterpret_cast<const Node*>(internals_dev), (uint32_t)n_internals,
            reinterpret_cast<const Attrib*>(attribs_dev), reinterpret_cast<NormalBound*>(out_dev));
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) return cuda_fail(e, "pz_normal_bounds");
    clear_error();
    return PZ_OK;
}

extern "C" size_t pz_path_cuts_scratch_bytes(int K, uint32_t frontier_capacity)
{
    if (K < 1 || K > kMaxK) return 0;
    return kHeader + 2 * (((size_t)frontier_capacity * entry_bytes(K) + 255) & ~(size_t)255);
}

template <int K>
static cudaError_t launch_round(const CutArgs& a, int directed, cudaStream_t s)
{
    const int grid = num_sms() * 8;
    if (directed) k_cuts_round<K, DR><<<grid, kBlock, 0, s>>>(a);
    else k_cuts_round<K, RN><<<grid, kBlock, 0, s>>>(a);
    return cudaGetLastError();
}

extern "C" int pz_path_cuts(int K, uint32_t events, float eta, pz_float3 p_beg, const pz_float3* p_end_dev,
                            uint32_t n_queries, const pz_internal_node* internals_dev, const pz_normal_bound* nbs_dev,
                            const pz_triangle* triangles_dev, const pz_triangle_attrib* attribs_dev,
                            const uint32_t* root_dev, int directed_rounding, uint32_t* tuples_dev,
                            uint32_t tuple_capacity, uint64_t* n_tuples_out, uint64_t* node_tuples_out,
                            void* scratch_dev, size_t scratch_bytes, pz_stream_t stream)
{
    if (K < 1 || K > kMaxK) return fail(PZ_ERR_INVALID_ARGUMENT, "pz_path_cuts: K must be 1..4 (got %d)", K);
    if (!n_tuples_out) return fail(PZ_ERR_INVALID_ARGUMENT, "pz_path_cuts: n_tuples_out is required");
    *n_tuples_out = 0;
    if (node_tuples_out) *node_tuples_out = 0;
    if (n_queries == 0) { clear_error(); return PZ_OK; }
    if (!p_end_dev || !internals_dev || !nbs_dev || !triangles_dev || !attribs_dev || !root_dev || !scratch_dev ||
        (tuple_capacity > 0 && !tuples_dev))
        return fail(PZ_ERR_INVALID_ARGUMENT, "pz_path_cuts: null buffer");
    if (scratch_bytes < pz_path_cuts_scratch_bytes(K, n_queries))
        return fail(PZ_ERR_SCRATCH_TOO_SMALL, "pz_path_cuts: scratch %zu < %zu (frontier must hold the queries)",
                    scratch_bytes, pz_path_cuts_scratch_bytes(K, n_queries));
    if (reinterpret_cast<uintptr_t>(scratch_dev) & 255)
        return fail(PZ_ERR_INVALID_ARGUMENT, "pz_path_cuts: scratch needs 256-byte alignment");
    // frontier capacity from the scratch size
    const size_t frontBytes = ((scratch_bytes - kHeader) / 2) & ~(size_t)15;
    const uint32_t frontCap = (uint32_t)std::min<size_t>(frontBytes / entry_bytes(K), 0xFFFFFFFFu);
    char* base = static_cast<char*>(scratch_dev);
    uint32_t* status = reinterpret_cast<uint32_t*>(base);
    unsigned long long* counts = reinterpret_cast<unsigned long long*>(base + 8);  // two frontier counts
    unsigned long long* nTup = reinterpret_cast<unsigned long long*>(base + 24);
    uint32_t* fronts[2] = {reinterpret_cast<uint32_t*>(base + kHeader),
                           reinterpret_cast<uint32_t*>(base + kHeader + frontBytes)};
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);

    CutArgs a;
    a.K = K;
    a.events = events;
    a.eta = eta;
    a.pBeg = make_float3(p_beg.x, p_beg.y, p_beg.z);
    a.pEnd = reinterpret_cast<const float3*>(p_end_dev);
    a.nQueries = n_queries;
    a.nodes = reinterpret_cast<const Node*>(internals_dev);
    a.nbs = reinterpret_cast<const NormalBound*>(nbs_dev);
    a.tris = reinterpret_cast<const Tri*>(triangles_dev);
    a.attribs = reinterpret_cast<const Attrib*>(attribs_dev);
    a.root = root_dev;
    a.frontCapacity = frontCap;  // >= n_queries (checked above)
    a.tuples = tuples_dev;
    a.nTuples = nTup;
    a.tupleCapacity = tuple_capacity;
    a.status = status;

    cudaError_t e = cudaMemsetAsync(base, 0, kHeader, s);
    if (e != cudaSuccess) return cuda_fail(e, "pz_path_cuts: clear");
    a.frontOut = fronts[0];
    a.countOut = &counts[0];
    k_cuts_init<<<(n_queries + kBlock - 1) / kBlock, kBlock, 0, s>>>(a);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "pz_path_cuts: init");
    uint64_t visited = 0;
    unsigned long long hostCount = n_queries;
    int cur = 0;
    // level by level; every round descends one node of every surviving tuple, so the
    // number of rounds is at most K times the BVH depth
    for (int round = 0; hostCount > 0; round++) {
        if (round > 4096) return fail(PZ_ERR_DEVICE, "pz_path_cuts: no end after 4096 levels");
        visited += std::min<unsigned long long>(hostCount, a.frontCapacity);
        a.frontIn = fronts[cur];
        a.countIn = &counts[cur];
        a.frontOut = fronts[cur ^ 1];
        a.countOut = &counts[cur ^ 1];
        e = cudaMemsetAsync(&counts[cur ^ 1], 0, sizeof(unsigned long long), s);
        if (e != cudaSuccess) return cuda_fail(e, "pz_path_cuts: clear count");
        switch (K) {
            case 1: e = launch_round<1>(a, directed_rounding, s); break;
            case 2: e = launch_round<2>(a, directed_rounding, s); break;
            case 3: e = launch_round<3>(a, directed_rounding, s); break;
            default: e = launch_round<4>(a, directed_rounding, s); break;
        }
        if (e != cudaSuccess) return cuda_fail(e, "pz_path_cuts: round");
        e = cudaMemcpyAsync(&hostCount, &counts[cur ^ 1], sizeof(hostCount), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cuda_fail(e, "pz_path_cuts: frontier count");
        cur ^= 1;
    }
    uint32_t st = 0;
    unsigned long long nt = 0;
    e = cudaMemcpyAsync(&st, status, sizeof(st), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&nt, nTup, sizeof(nt), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(e, "pz_path_cuts: results");
    *n_tuples_out = nt;
    if (node_tuples_out) *node_tuples_out = visited;
    if (st & kErrCapacity)
        return fail(PZ_ERR_DEVICE, "pz_path_cuts: capacity exceeded (%llu tuples for %u slots, or the frontier)",
                    (unsigned long long)nt, tuple_capacity);
    clear_error();
    return PZ_OK;
}
