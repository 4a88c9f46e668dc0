// pz_subdiv.cu -- per-tuple parametric-domain subdivision under affine bounds, and the
// Newton solve in the boxes that survive.
//
// No reference counterpart.  The reference solves each admissible tuple once, from one
// start (main.cpp:1052, solveConstraints<K>, pk.h:466-592), and so finds at most one root
// per tuple.  Here the domain of every tuple -- its 2K barycentrics, the unit box
// [0,1]^2K -- is bisected level by level: split t halves dimension t mod 2K, so a box is
// named by its depth and the bits of its bisection path.  A box is dropped when
//   - it lies outside a triangle (u_lo + v_lo > 1 for some vertex), or
//   - an affine bound of the specular constraint the Newton solver drives to zero
//     (the cross product of the outgoing direction with the reflected / refracted one,
//     taken on the side of the shading normal the solver takes) excludes zero in some
//     component: no root lies in the box, or
//   - the sign pattern of the two cosines at some vertex rules out the event over the
//     whole box, which contributableThroughput (pk.h:760-842) would reject, or
//   - the joint linear test finds no root: with two residual components per vertex (the
//     ones off the outgoing direction's largest axis) the affine forms are a 2K x 2K
//     linear system in the box parameters plus bounded remainders, and a Krawczyk-style
//     enclosure of its solutions misses the box.
// A box stops splitting at the depth limit, or when every bounded residual component is
// narrower than eps (the bound no longer tightens usefully).  Its centre then starts the
// reference's Newton solve, once per wavelength bin that may hold a root there.  A root
// is kept when
//   - the solve converged,
//   - the root lies in that box (half-open boxes: every root has one owner box, so no
//     root is reported twice),
//   - contributableThroughput, visibility included, is positive.
// The wavelength bins share one subdivision: eta^2 - 1 over the range of the bins' values
// is one more noise symbol of the bound, so a box that survives for any bin survives.  At
// a leaf, each bin's value of that symbol is substituted into the residual forms and the
// joint linear test, and a bin for which either then excludes a root gets no Newton solve.
//
// Affine forms: x = c + sum_i x_i e_i + r e_err with |e_i|, |e_err| <= 1; the noise
// symbols e_i are the box's 2K parameters and eta^2 - 1.  Central and linear coefficients are rounded
// to nearest; each rounding error, and each nonlinear remainder, goes into the radius r
// with upward rounding, so the bound encloses the constraint in exact arithmetic.  The
// unit is built with -fmad=false, so the CPU oracle can repeat every operation.
//
// Kernels: k_sub_init (one entry per tuple), k_sub_round (one launch per depth; a thread
// per box: bound, cull, split or retire to the leaf list; warp-aggregated appends),
// k_sub_leaf_test (a thread per leaf: the per-bin test, surviving (leaf, bin) pairs to a
// compact solve list), k_sub_leaf_solve (a thread per pair: Newton, ownership, throughput,
// root output), k_sub_contribute (a thread per root: dAdw and the binned spectral image).
// The rounds read their input count on the device: no host synchronisation between
// launches.
#include <algorithm>

#include "pz_capi_internal.h"
#include "pz_common.cuh"
#include "pz_frame.cuh"
#include "pz_solver.cuh"

namespace pz {
namespace subdiv {

using solver::Chain;
using solver::V3;

constexpr int kBlock = 256;
constexpr int kMaxDepth = 20;  // path bits in an entry
constexpr int kMaxBins = 256;
constexpr uint32_t kPathMask = (1u << kMaxDepth) - 1u;

enum : int {
    kStTested = 0, kStCulled, kStExcluded, kStSolves, kStConverged, kStOutside, kStRoots, kStPolished, kNumStats
};

// ---------------------------------------------------------------- affine forms
// Rounding error of one round-to-nearest result r: at most |r| 2^-24 (normal) or 2^-150.
PZ_D float rerr(float r) { return __fadd_ru(__fmul_ru(fabsf(r), 0x1p-24f), 0x1p-149f); }

template <int N> struct Af {
    float c, x[N], r;
};
template <int N> struct Af3 {
    Af<N> x, y, z;
};

template <int N> PZ_D Af<N> af_const(float v)
{
    Af<N> o;
    o.c = v;
#pragma unroll
    for (int i = 0; i < N; i++) o.x[i] = 0.0f;
    o.r = 0.0f;
    return o;
}

template <int N> PZ_D Af<N> af_add(const Af<N>& a, const Af<N>& b)
{
    Af<N> o;
    o.c = __fadd_rn(a.c, b.c);
    float r = __fadd_ru(__fadd_ru(a.r, b.r), rerr(o.c));
#pragma unroll
    for (int i = 0; i < N; i++) {
        o.x[i] = __fadd_rn(a.x[i], b.x[i]);
        r = __fadd_ru(r, rerr(o.x[i]));
    }
    o.r = r;
    return o;
}

template <int N> PZ_D Af<N> af_sub(const Af<N>& a, const Af<N>& b)
{
    Af<N> o;
    o.c = __fsub_rn(a.c, b.c);
    float r = __fadd_ru(__fadd_ru(a.r, b.r), rerr(o.c));
#pragma unroll
    for (int i = 0; i < N; i++) {
        o.x[i] = __fsub_rn(a.x[i], b.x[i]);
        r = __fadd_ru(r, rerr(o.x[i]));
    }
    o.r = r;
    return o;
}

template <int N> PZ_D Af<N> af_neg(const Af<N>& a)
{
    Af<N> o;
    o.c = -a.c;
#pragma unroll
    for (int i = 0; i < N; i++) o.x[i] = -a.x[i];
    o.r = a.r;
    return o;
}

// sum |x_i| + r, rounded up
template <int N> PZ_D float af_rad(const Af<N>& a)
{
    float s = a.r;
#pragma unroll
    for (int i = 0; i < N; i++) s = __fadd_ru(s, fabsf(a.x[i]));
    return s;
}
template <int N> PZ_D float af_lo(const Af<N>& a) { return __fsub_rd(a.c, af_rad(a)); }
template <int N> PZ_D float af_hi(const Af<N>& a) { return __fadd_ru(a.c, af_rad(a)); }

// a*b = ac bc + ac (Lb + Eb) + bc (La + Ea) + (La + Ea)(Lb + Eb); the linear parts are
// kept, the rest is bounded by |ac| rb_err + |bc| ra_err + rad(a) rad(b).
template <int N> PZ_D Af<N> af_mul(const Af<N>& a, const Af<N>& b)
{
    Af<N> o;
    o.c = __fmul_rn(a.c, b.c);
    float r = rerr(o.c);
    float ra = a.r, rb = b.r;
#pragma unroll
    for (int i = 0; i < N; i++) {
        const float p = __fmul_rn(a.c, b.x[i]), q = __fmul_rn(b.c, a.x[i]);
        o.x[i] = __fadd_rn(p, q);
        r = __fadd_ru(r, __fadd_ru(__fadd_ru(rerr(p), rerr(q)), rerr(o.x[i])));
        ra = __fadd_ru(ra, fabsf(a.x[i]));
        rb = __fadd_ru(rb, fabsf(b.x[i]));
    }
    r = __fadd_ru(r, __fmul_ru(fabsf(a.c), b.r));
    r = __fadd_ru(r, __fmul_ru(fabsf(b.c), a.r));
    o.r = __fadd_ru(r, __fmul_ru(ra, rb));
    return o;
}

// a * s for an exact float s
template <int N> PZ_D Af<N> af_scale(const Af<N>& a, float s)
{
    Af<N> o;
    o.c = __fmul_rn(a.c, s);
    float r = __fadd_ru(__fmul_ru(a.r, fabsf(s)), rerr(o.c));
#pragma unroll
    for (int i = 0; i < N; i++) {
        o.x[i] = __fmul_rn(a.x[i], s);
        r = __fadd_ru(r, rerr(o.x[i]));
    }
    o.r = r;
    return o;
}

// a + s for an exact float s
template <int N> PZ_D Af<N> af_addc(const Af<N>& a, float s)
{
    Af<N> o = a;
    o.c = __fadd_rn(a.c, s);
    o.r = __fadd_ru(a.r, rerr(o.c));
    return o;
}

// sqrt on [lo, hi], lo >= 0, by the min-range linearisation sqrt(x) = alpha x + d(x),
// alpha <= 1 / (2 sqrt(hi)) so that d is nondecreasing on [lo, hi] and lies in
// [d(lo), d(hi)] = zeta -+ delta.
template <int N> PZ_D Af<N> af_sqrt(const Af<N>& a)
{
    const float lo = fmaxf(af_lo(a), 0.0f), hi = af_hi(a);
    if (!(hi > 0.0f)) return af_const<N>(0.0f);
    const float sh = __fsqrt_ru(hi);
    const float alpha = __fdiv_rd(1.0f, __fmul_ru(2.0f, sh));
    const float dlo = __fsub_rd(__fsqrt_rd(lo), __fmul_ru(alpha, lo));
    const float dhi = __fsub_ru(sh, __fmul_rd(alpha, hi));
    const float zeta = __fmul_rn(__fadd_rn(dlo, dhi), 0.5f);
    const float delta = fmaxf(__fsub_ru(dhi, zeta), __fsub_ru(zeta, dlo));
    Af<N> o = af_addc(af_scale(a, alpha), zeta);
    o.r = __fadd_ru(o.r, delta);
    return o;
}

template <int N> PZ_D Af3<N> af3_const(float3 v) { return Af3<N>{af_const<N>(v.x), af_const<N>(v.y), af_const<N>(v.z)}; }
template <int N> PZ_D Af3<N> af3_sub(const Af3<N>& a, const Af3<N>& b)
{
    return Af3<N>{af_sub(a.x, b.x), af_sub(a.y, b.y), af_sub(a.z, b.z)};
}
template <int N> PZ_D Af3<N> af3_add(const Af3<N>& a, const Af3<N>& b)
{
    return Af3<N>{af_add(a.x, b.x), af_add(a.y, b.y), af_add(a.z, b.z)};
}
template <int N> PZ_D Af3<N> af3_mul(const Af3<N>& a, const Af<N>& s)
{
    return Af3<N>{af_mul(a.x, s), af_mul(a.y, s), af_mul(a.z, s)};
}
template <int N> PZ_D Af<N> af3_dot(const Af3<N>& a, const Af3<N>& b)
{
    return af_add(af_add(af_mul(a.x, b.x), af_mul(a.y, b.y)), af_mul(a.z, b.z));
}
template <int N> PZ_D Af3<N> af3_cross(const Af3<N>& a, const Af3<N>& b)
{
    return Af3<N>{af_sub(af_mul(a.y, b.z), af_mul(a.z, b.y)), af_sub(af_mul(a.z, b.x), af_mul(a.x, b.z)),
                  af_sub(af_mul(a.x, b.y), af_mul(a.y, b.x))};
}
// p0 + e0 u + e1 v (the Newton solver's vertex and shading-normal interpolation)
template <int N> PZ_D Af<N> af_lin(float p0, float e0, float e1, const Af<N>& u, const Af<N>& v)
{
    return af_add(af_addc(af_scale(u, e0), p0), af_scale(v, e1));
}
template <int N> PZ_D Af3<N> af3_lin(float3 p0, float3 e0, float3 e1, const Af<N>& u, const Af<N>& v)
{
    return Af3<N>{af_lin(p0.x, e0.x, e1.x, u, v), af_lin(p0.y, e0.y, e1.y, u, v), af_lin(p0.z, e0.z, e1.z, u, v)};
}

// ---------------------------------------------------------------- boxes
// Box of depth d with bisection path `path`: dimension j is halved at splits j, j + N,
// j + 2N, ... < d; bit t of the path is the half taken at split t.
template <int N> PZ_D void box_bounds(uint32_t path, int depth, float* lo, float* hi)
{
#pragma unroll
    for (int j = 0; j < N; j++) {
        float l = 0.0f, w = 1.0f;
        for (int t = j; t < depth; t += N) {
            w *= 0.5f;
            if ((path >> t) & 1u) l += w;
        }
        lo[j] = l;
        hi[j] = l + w;
    }
}

enum Verdict : int { kCull = 0, kSplit = 1, kLeaf = 2 };

// The residual of one vertex over a box, for the per-bin test of the leaves: per component
// the centre, the radius without the eta^2 - 1 symbol, and that symbol's coefficient.
struct VertexForms {
    bool valid;
    float c[3], rad[3], xe[3];
};

// Joint linear test over the box.  Rows j = 0 .. n-1 model the residual as
// c0_j + sum_l A_jl e_l + d_j with |d_j| <= r_j and the box parameters e in [-1, 1]^n.  For
// any matrix Y, a solution satisfies e = -Y c0 - Y d + (I - Y A) e, so e_i lies within
// -(Y c0)_i -+ (sum_j |Y_ij| r_j + sum_l |(I - Y A)_il|).  When that interval misses
// [-1, 1] for some i there is no root in the box.  Y is A's inverse by Gauss-Jordan
// elimination rounded to nearest (any Y keeps the test sound; a singular or non-finite
// one skips it); every term of the enclosure is rounded outward.
template <int n> struct LinearTest {
    bool ok;            // false: A singular or Y not finite (no test)
    float Y[n][n];      // approximate inverse of A
    float e[n];         // sum_l |(I - Y A)_il|, rounded up
};

template <int n>
PZ_D void linear_prepare(LinearTest<n>& T, const float (&A)[n][n])
{
    float M[n][2 * n];
#pragma unroll
    for (int i = 0; i < n; i++)
#pragma unroll
        for (int j = 0; j < 2 * n; j++) M[i][j] = j < n ? A[i][j] : (j - n == i ? 1.0f : 0.0f);
    T.ok = false;
#pragma unroll
    for (int col = 0; col < n; col++) {
        int piv = col;
        float best = fabsf(M[col][col]);
#pragma unroll
        for (int i = col + 1; i < n; i++)
            if (fabsf(M[i][col]) > best) {
                best = fabsf(M[i][col]);
                piv = i;
            }
#pragma unroll
        for (int i = col + 1; i < n; i++) {  // swap rows col and piv (constant indices: registers)
            if (i != piv) continue;
#pragma unroll
            for (int j = 0; j < 2 * n; j++) {
                const float t = M[col][j];
                M[col][j] = M[i][j];
                M[i][j] = t;
            }
        }
        if (!(fabsf(M[col][col]) > 0.0f)) return;
        const float inv = __fdiv_rn(1.0f, M[col][col]);
#pragma unroll
        for (int j = 0; j < 2 * n; j++) M[col][j] = __fmul_rn(M[col][j], inv);
#pragma unroll
        for (int i = 0; i < n; i++) {
            if (i == col) continue;
            const float f = M[i][col];
#pragma unroll
            for (int j = 0; j < 2 * n; j++) M[i][j] = __fsub_rn(M[i][j], __fmul_rn(f, M[col][j]));
        }
    }
#pragma unroll
    for (int i = 0; i < n; i++)
#pragma unroll
        for (int j = 0; j < n; j++) {
            if (!isfinite(M[i][n + j])) return;
            T.Y[i][j] = M[i][n + j];
        }
#pragma unroll
    for (int i = 0; i < n; i++) {
        float rad = 0.0f;
#pragma unroll
        for (int l = 0; l < n; l++) {
            float sLo = 0.0f, sHi = 0.0f;
#pragma unroll
            for (int j = 0; j < n; j++) {
                sLo = __fadd_rd(sLo, __fmul_rd(T.Y[i][j], A[j][l]));
                sHi = __fadd_ru(sHi, __fmul_ru(T.Y[i][j], A[j][l]));
            }
            const float d = i == l ? 1.0f : 0.0f;
            rad = __fadd_ru(rad, fmaxf(__fsub_ru(sHi, d), __fsub_ru(d, sLo)));
        }
        T.e[i] = rad;
    }
    T.ok = true;
}

// True when no root lies in the box, for rows with centres c0 and radii r.
template <int n>
PZ_D bool linear_excludes(const LinearTest<n>& T, const float (&c0)[n], const float (&r)[n])
{
    if (!T.ok) return false;
#pragma unroll
    for (int i = 0; i < n; i++) {
        float lo = 0.0f, hi = 0.0f, rad = T.e[i];
#pragma unroll
        for (int j = 0; j < n; j++) {
            const float y = T.Y[i][j];
            lo = __fadd_rd(lo, __fmul_rd(-y, c0[j]));
            hi = __fadd_ru(hi, __fmul_ru(-y, c0[j]));
            rad = __fadd_ru(rad, __fmul_ru(fabsf(y), r[j]));
        }
        if (__fsub_rd(lo, rad) > 1.0f || __fadd_ru(hi, rad) < -1.0f) return true;
    }
    return false;
}

// The joint test's rows of a leaf, kept for the per-bin tests: the prepared inverse, and
// per row the centre, the eta^2 - 1 coefficient and the nonlinear radius.
template <int K> struct LinearRows {
    bool valid;
    LinearTest<2 * K> test;
    float c[2 * K], xe[2 * K], r[2 * K];
};

// The joint test for one bin: the bin's eta symbol [elo, ehi] substituted into every row
// (its spread goes into the radius).
template <int K>
PZ_D bool bin_linear_excludes(const LinearRows<K>& L, float elo, float ehi)
{
    if (!L.valid) return false;
    float c0[2 * K], r[2 * K];
#pragma unroll
    for (int j = 0; j < 2 * K; j++) {
        const float pl = fminf(__fmul_rd(L.xe[j], elo), __fmul_rd(L.xe[j], ehi));
        const float ph = fmaxf(__fmul_ru(L.xe[j], elo), __fmul_ru(L.xe[j], ehi));
        const float cl = __fadd_rd(L.c[j], pl), ch = __fadd_ru(L.c[j], ph);
        c0[j] = __fmul_rn(__fadd_rn(cl, ch), 0.5f);
        r[j] = __fadd_ru(L.r[j], fmaxf(__fsub_ru(ch, c0[j]), __fsub_ru(c0[j], cl)));
    }
    return linear_excludes<2 * K>(L.test, c0, r);
}

// The bound of one box.  Noise symbols 0 .. 2K-1 are the box's parameters, symbol 2K is
// eta^2 - 1 over the bins (em1).  forms (may be null) receives each vertex's residual.
template <int K>
PZ_D int bound_box(const Chain<K>& ch, float3 pBeg, float3 pEnd, uint32_t events, const Af<2 * K + 1>& em1,
                   const float* lo, const float* hi, float eps, VertexForms* forms = nullptr,
                   LinearRows<K>* rows = nullptr)
{
    constexpr int N = 2 * K + 1;
#pragma unroll
    for (int k = 0; k < K; k++)
        if (__fadd_rd(lo[2 * k], lo[2 * k + 1]) > 1.0f) return kCull;  // outside the triangle
    Af3<N> X[K + 2], Nrm[K];
    X[0] = af3_const<N>(pBeg);
    X[K + 1] = af3_const<N>(pEnd);
#pragma unroll
    for (int k = 0; k < K; k++) {
        Af<N> u = af_const<N>(__fmul_rn(__fadd_rn(lo[2 * k], hi[2 * k]), 0.5f));
        Af<N> v = af_const<N>(__fmul_rn(__fadd_rn(lo[2 * k + 1], hi[2 * k + 1]), 0.5f));
        u.x[2 * k] = __fmul_rn(__fsub_rn(hi[2 * k], lo[2 * k]), 0.5f);
        v.x[2 * k + 1] = __fmul_rn(__fsub_rn(hi[2 * k + 1], lo[2 * k + 1]), 0.5f);
        X[k + 1] = af3_lin(ch.v0[k], ch.e0[k], ch.e1[k], u, v);
        Nrm[k] = af3_lin(ch.n0[k], ch.ne0[k], ch.ne1[k], u, v);
    }
    bool resolved = true, linear = true;
    float lc0[2 * K], lA[2 * K][2 * K], lr[2 * K];  // two residual rows per vertex for the joint test
    float lxe[2 * K], lrn[2 * K];                     // their eta coefficients and nonlinear radii
#pragma unroll
    for (int k = 0; k < K; k++) {
        if (forms) forms[k].valid = false;
        Af3<N> wi = af3_sub(X[k], X[k + 1]);
        Af3<N> wo = af3_sub(X[k + 2], X[k + 1]);
        const Af3<N>& n = Nrm[k];
        const Af<N> s = af3_dot(wi, n), t = af3_dot(wo, n);
        const float sl = af_lo(s), sh = af_hi(s), tl = af_lo(t), th = af_hi(t);
        const bool refract = (events >> k) & 1u;
        // the event needs (wi.n)(wo.n) <= 0 (T) or > 0 (R) somewhere in the box
        if (refract ? ((sl > 0.0f && tl > 0.0f) || (sh < 0.0f && th < 0.0f))
                    : ((sl >= 0.0f && th <= 0.0f) || (sh <= 0.0f && tl >= 0.0f)))
            return kCull;
        // the solver refracts / reflects the direction on the normal's side of the surface
        if (sh < 0.0f) {
            const Af3<N> tmp = wi;
            wi = wo;
            wo = tmp;
        } else if (!(sl >= 0.0f)) {
            resolved = false;  // the side changes inside the box: no bound at this vertex
            linear = false;
            continue;
        }
        const Af<N> NoN = af3_dot(n, n);
        const Af<N> WIoN = af3_dot(wi, n);
        Af3<N> w;
        if (refract) {
            // -wi (n.n) + n ((wi.n) - sqrt((n.n)(wi.wi)(eta^2 - 1) + (wi.n)^2)), pk.h:181-200
            const Af<N> WoW = af3_dot(wi, wi);
            const Af<N> kk = af_add(af_mul(af_mul(NoN, WoW), em1), af_mul(WIoN, WIoN));
            if (!(af_lo(kk) >= 0.0f)) {  // total internal reflection in part of the box
                resolved = false;
                linear = false;
                continue;
            }
            const Af<N> g = af_sub(WIoN, af_sqrt(kk));
            w = af3_add(Af3<N>{af_neg(af_mul(wi.x, NoN)), af_neg(af_mul(wi.y, NoN)), af_neg(af_mul(wi.z, NoN))},
                        af3_mul(n, g));
        } else {
            // (n.n) times the reflection n (wi.n) 2 / (n.n) - wi: the same zeros for n != 0
            if (!(af_lo(NoN) > 0.0f)) {
                resolved = false;
                linear = false;
                continue;
            }
            const Af<N> d2 = af_scale(WIoN, 2.0f);
            w = af3_sub(af3_mul(n, d2), af3_mul(wi, NoN));
        }
        const Af3<N> c = af3_cross(wo, w);
        const Af<N>* cc[3] = {&c.x, &c.y, &c.z};
#pragma unroll
        for (int j = 0; j < 3; j++) {
            const float l = af_lo(*cc[j]), h = af_hi(*cc[j]);
            if (l > 0.0f || h < 0.0f) return kCull;
            resolved = resolved && __fsub_ru(h, l) < eps;
            if (forms) {
                float r = cc[j]->r;
#pragma unroll
                for (int i = 0; i < N - 1; i++) r = __fadd_ru(r, fabsf(cc[j]->x[i]));
                forms[k].c[j] = cc[j]->c;
                forms[k].rad[j] = r;
                forms[k].xe[j] = cc[j]->x[N - 1];
            }
        }
        if (forms) forms[k].valid = true;
        // the two components of c = wo x w that do not lie along wo's largest axis (that
        // one is about zero everywhere), for the joint test; eta^2 - 1 goes into the radius
        const float ax = fabsf(wo.x.c), ay = fabsf(wo.y.c), az = fabsf(wo.z.c);
        const int drop = (ax >= ay && ax >= az) ? 0 : (ay >= az ? 1 : 2);
        const Af<N>& ra = drop == 0 ? c.y : c.x;  // the first kept component
        const Af<N>& rb = drop == 2 ? c.y : c.z;  // the second
        lc0[2 * k] = ra.c;
        lc0[2 * k + 1] = rb.c;
#pragma unroll
        for (int i = 0; i < N - 1; i++) {
            lA[2 * k][i] = ra.x[i];
            lA[2 * k + 1][i] = rb.x[i];
        }
        lr[2 * k] = __fadd_ru(ra.r, fabsf(ra.x[N - 1]));
        lr[2 * k + 1] = __fadd_ru(rb.r, fabsf(rb.x[N - 1]));
        lxe[2 * k] = ra.x[N - 1];
        lxe[2 * k + 1] = rb.x[N - 1];
        lrn[2 * k] = ra.r;
        lrn[2 * k + 1] = rb.r;
    }
    if (linear) {
        LinearTest<2 * K> T;
        linear_prepare<2 * K>(T, lA);
        if (linear_excludes<2 * K>(T, lc0, lr)) return kCull;
        if (rows) {
            rows->test = T;
#pragma unroll
            for (int j = 0; j < 2 * K; j++) {
                rows->c[j] = lc0[j];
                rows->xe[j] = lxe[j];
                rows->r[j] = lrn[j];
            }
        }
    }
    if (rows) rows->valid = linear;
    return resolved ? kLeaf : kSplit;
}

// eta^2 - 1 over the bins as an affine form: centre + radius * (its own noise symbol)
template <int M> PZ_D Af<M> em1_form(float mLo, float mHi)
{
    Af<M> e = af_const<M>(__fmul_rn(__fadd_rn(mLo, mHi), 0.5f));
    e.x[M - 1] = fmaxf(__fsub_ru(mHi, e.c), __fsub_ru(e.c, mLo));
    return e;
}

// The eta symbol's value for the bin value m of eta^2 - 1: (m - centre) / radius, as an
// interval [*elo, *ehi].
template <int M> PZ_D void bin_symbol(const Af<M>& em1, float m, float* elo, float* ehi)
{
    const float rad = em1.x[M - 1];
    *elo = *ehi = 0.0f;
    if (rad > 0.0f) {
        *elo = __fdiv_rd(__fsub_rd(m, em1.c), rad);
        *ehi = __fdiv_ru(__fsub_ru(m, em1.c), rad);
    }
}

// Can a root for a bin lie in the box?  Substitutes the bin's value of the eta symbol,
// [elo, ehi], into every vertex's residual components; false when some component's range
// then excludes zero.
template <int K>
PZ_D bool bin_may_hold_root(const VertexForms* forms, float elo, float ehi)
{
#pragma unroll
    for (int k = 0; k < K; k++) {
        if (!forms[k].valid) continue;
#pragma unroll
        for (int j = 0; j < 3; j++) {
            const float xe = forms[k].xe[j];
            const float pl = fminf(__fmul_rd(xe, elo), __fmul_rd(xe, ehi));
            const float ph = fmaxf(__fmul_ru(xe, elo), __fmul_ru(xe, ehi));
            const float l = __fsub_rd(__fadd_rd(forms[k].c[j], pl), forms[k].rad[j]);
            const float h = __fadd_ru(__fadd_ru(forms[k].c[j], ph), forms[k].rad[j]);
            if (l > 0.0f || h < 0.0f) return false;
        }
    }
    return true;
}

// ---------------------------------------------------------------- kernels
struct SubArgs {
    uint32_t events;
    float3 pBeg;
    const float3* pEnd;
    const uint32_t* tuples;  // (1 + K) u32 per row: query, triangles
    uint32_t nRows;
    const float* etas;
    uint32_t nBins;
    int maxDepth;
    float eps;
    int maxIterations;
    float costTolerance;
    int warmUp;
    int polish;
    const Tri* tris;  // the triangles the tuple rows index
    const Attrib* attribs;
    const Node* nodes;  // visibility: the scene's BVH and triangles
    const Tri* sceneTris;
    const uint32_t* root;
    uint64_t capacity;  // entries per frontier and in the leaf list
    float* em1;         // [2]: range of eta^2 - 1 over the bins
    uint64_t* leaves;
    unsigned long long* nLeaves;
    uint64_t* items;  // (leaf, bin) pairs to solve, in the two frontiers' space
    unsigned long long* nItems;
    uint64_t itemCapacity;
    pz_specular_root* roots;
    unsigned long long* nRoots;
    uint64_t rootCapacity;
    unsigned long long* stats;
    uint32_t* status;
    // box queue of the persistent subdivision kernel: a ring of ringCapacity entries and its
    // claim / reserve / outstanding counters
    uint64_t* ring;
    uint64_t ringCapacity;
    unsigned long long* qHead;     // entries claimed by consumers
    unsigned long long* qTail;     // entries reserved by producers
    unsigned long long* qPending;  // boxes pushed and not yet finished
};

// entry: row << 32 | depth << 20 | path
PZ_D uint64_t make_entry(uint32_t row, int depth, uint32_t path)
{
    return ((uint64_t)row << 32) | ((uint64_t)depth << kMaxDepth) | (path & kPathMask);
}

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

// Sum of v over the active lanes (*total) and this lane's exclusive prefix of it, by one
// shuffle per lane of the warp (correct for any set of active lanes).
PZ_D uint32_t warp_prefix(uint32_t active, uint32_t v, uint32_t* total)
{
    const int lane = (int)(threadIdx.x & 31);
    uint32_t pre = 0, tot = 0;
#pragma unroll
    for (int j = 0; j < 32; j++) {
        const uint32_t x = __shfl_sync(active, v, j);
        if ((active >> j) & 1u) {
            tot += x;
            if (j < lane) pre += x;
        }
    }
    *total = tot;
    return pre;
}

// warp-aggregated reservation of n consecutive slots per lane: one atomic per warp
PZ_D unsigned long long warp_reserve(unsigned long long* counter, uint32_t n)
{
    const uint32_t active = __activemask();
    const int leader = __ffs(active) - 1;
    uint32_t total;
    const uint32_t pre = warp_prefix(active, n, &total);
    unsigned long long base = 0;
    if ((int)(threadIdx.x & 31) == leader && total) base = atomicAdd(counter, (unsigned long long)total);
    base = __shfl_sync(active, base, leader);
    return base + pre;
}

PZ_D void warp_sum(unsigned long long* stat, uint32_t v)
{
    const uint32_t active = __activemask();
    uint32_t total;
    warp_prefix(active, v, &total);
    if ((int)(threadIdx.x & 31) == __ffs(active) - 1 && total) atomicAdd(stat, (unsigned long long)total);
}

template <int K>
PZ_D void load_row(Chain<K>& ch, const SubArgs& a, uint32_t row, uint32_t* q)
{
    const uint32_t* t = a.tuples + (size_t)row * (1 + K);
    int idx[K];
#pragma unroll
    for (int k = 0; k < K; k++) idx[k] = (int)__ldg(t + 1 + k);
    *q = __ldg(t);
    solver::load_chain<K>(ch, a.tris, a.attribs, idx);
}

// eta^2 - 1 over the bins, the way the solver forms it; then the first frontier
__global__ void k_sub_init(SubArgs a, uint64_t* front, unsigned long long* count)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        float lo = 0.0f, hi = 0.0f;
        for (uint32_t b = 0; b < a.nBins; b++) {
            const float e = a.etas[b];
            const float m = __fsub_rn(__fmul_rn(e, e), 1.0f);
            lo = b == 0 ? m : fminf(lo, m);
            hi = b == 0 ? m : fmaxf(hi, m);
        }
        a.em1[0] = lo;
        a.em1[1] = hi;
        *count = a.nRows;
    }
    const uint32_t row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row < a.nRows) front[row] = make_entry(row, 0, 0u);
}

template <int K>
__global__ void __launch_bounds__(kBlock) k_sub_round(SubArgs a, int depth, const uint64_t* __restrict__ frontIn,
                                                      const unsigned long long* countIn, uint64_t* __restrict__ frontOut,
                                                      unsigned long long* countOut)
{
    constexpr int N = 2 * K;
    const uint64_t nIn = min((uint64_t)*countIn, a.capacity);
    const Af<N + 1> em1 = em1_form<N + 1>(a.em1[0], a.em1[1]);
    const bool last = depth >= a.maxDepth;
    uint32_t tested = 0, culled = 0;
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nIn; e += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t ent = frontIn[e];
        const uint32_t row = (uint32_t)(ent >> 32), path = (uint32_t)ent & kPathMask;
        Chain<K> ch;
        uint32_t q;
        load_row<K>(ch, a, row, &q);
        float lo[N], hi[N];
        box_bounds<N>(path, depth, lo, hi);
        int v = bound_box<K>(ch, a.pBeg, a.pEnd[q], a.events, em1, lo, hi, a.eps);
        if (v == kSplit && last) v = kLeaf;
        tested++;
        culled += v == kCull;
        const unsigned long long ls = warp_append(a.nLeaves, v == kLeaf);
        if (v == kLeaf) {
            if (ls < a.capacity) a.leaves[ls] = make_entry(row, depth, path);
            else raise_error(a.status, kErrCapacity);
        }
        const unsigned long long s = warp_reserve(countOut, v == kSplit ? 2u : 0u);
        if (v == kSplit) {
            if (s + 1 < a.capacity) {
                frontOut[s] = make_entry(row, depth + 1, path);
                frontOut[s + 1] = make_entry(row, depth + 1, path | (1u << depth));
            } else {
                raise_error(a.status, kErrCapacity);
            }
        }
    }
    if (a.stats) {
        warp_sum(a.stats + kStTested, tested);
        warp_sum(a.stats + kStCulled, culled);
    }
}

// ---------------------------------------------------------------- persistent box queue
// Tuples whose domains need very different depths share one persistent kernel fed by a
// device-side queue (k_sub_queue below).  The queue is a ring of entries in the scratch's
// two frontier regions: a slot holds an entry with kQueued set and the lap of its index, or
// 0 when free.  A producer reserves indices on qTail and waits (bounded) until each slot is
// free before storing; a consumer claims indices on qHead and takes a slot once its entry
// (of the right lap) is stored, then frees it.  Every wait has an iteration limit (status
// kErrSpinLimit); a ring too small for the live boxes sets kErrCapacity.  Which warp bounds
// which box changes nothing: the leaves are a set (sorted by row afterwards), as with one
// launch per depth.
constexpr uint64_t kQueued = 1ull << 31;  // above the depth field of an entry
constexpr int kLapShift = 25;              // bits 25-30: the ring lap of the entry's index
constexpr uint64_t kLapMask = 63ull << kLapShift;
constexpr uint32_t kQueueSpin = 1u << 22;
static_assert(kMaxDepth + 5 <= kLapShift, "the lap bits sit above an entry's depth field");

// an entry as stored in ring slot i % cap: queued bit and the lap i / cap (mod 64), so that a
// consumer of index i never takes the entry of index i - cap still waiting in the slot
PZ_D uint64_t queued_entry(uint64_t ent, uint64_t index, uint64_t cap)
{
    return ent | kQueued | (((index / cap) & 63ull) << kLapShift);
}

PZ_D unsigned long long ld_volatile(const unsigned long long* p)
{
    return *reinterpret_cast<const volatile unsigned long long*>(p);
}

// the first boxes: one per row at depth 0, and the queue counters
__global__ void k_sub_queue_init(SubArgs a)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        float lo = 0.0f, hi = 0.0f;
        for (uint32_t b = 0; b < a.nBins; b++) {
            const float e = a.etas[b];
            const float m = __fsub_rn(__fmul_rn(e, e), 1.0f);
            lo = b == 0 ? m : fminf(lo, m);
            hi = b == 0 ? m : fmaxf(hi, m);
        }
        a.em1[0] = lo;
        a.em1[1] = hi;
        *a.qHead = 0;
        *a.qTail = a.nRows;
        *a.qPending = a.nRows;
    }
    const uint32_t row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row < a.nRows) a.ring[row] = queued_entry(make_entry(row, 0, 0u), row, a.ringCapacity);
}

constexpr int kLocal = 256;                 // entries of a warp's local box stack (shared memory)
#ifndef PZ_SUBDIV_LEND_ABOVE
#define PZ_SUBDIV_LEND_ABOVE 64
#endif
#ifndef PZ_SUBDIV_LEND_EVERY
#define PZ_SUBDIV_LEND_EVERY 1
#endif
constexpr int kDonateAbove = PZ_SUBDIV_LEND_ABOVE;  // a warp holding more lends boxes to the ring when it runs low
constexpr int kLendEvery = PZ_SUBDIV_LEND_EVERY;    // passes between two looks at the ring's level
constexpr uint64_t kNoClaim = ~0ull;

// Stores this lane's entry in the ring when `want`; all lanes of the warp call it.  False
// when the ring is full (kErrCapacity) or a wait for a free slot gave up.
PZ_D bool ring_push(const SubArgs& a, bool want, uint64_t ent)
{
    const unsigned long long i = warp_reserve(a.qTail, want ? 1u : 0u);
    bool ok = true;
    if (want) {
        const uint64_t cap = a.ringCapacity;
        volatile uint64_t* ring = a.ring;
        if (i >= ld_volatile(a.qHead) + cap) {
            // the slot's previous entry (index i - cap) is not even claimed: the ring is full
            raise_error(a.status, kErrCapacity);
            ok = false;
        } else {
            const uint64_t slot = i % cap;
            uint32_t spin = 0;
            while (ring[slot] != 0ull) {
                if (++spin >= kQueueSpin) {
                    ok = false;
                    break;
                }
                __nanosleep(64);
            }
            if (ok) ring[slot] = queued_entry(ent, i, cap);
        }
    }
    return __all_sync(0xFFFFFFFFu, ok);
}

// Persistent subdivision: each warp bounds up to 32 boxes per pass, taken from its own stack
// of boxes in shared memory (newest first: depth first, so the stack stays short and a pass
// mostly holds boxes of one tuple), else from the ring.  Children go to the warp's stack;
// what does not fit goes to the ring, and a warp holding many boxes lends its oldest ones to
// the ring whenever the ring runs low, so that idle warps share a deep tuple's boxes.
// Claims on the ring are taken with one atomic add per warp; a claimed slot whose entry is
// not stored yet is checked again on the next pass while the lane's other work goes on (no
// lane waits on another warp's progress except for a free slot).  qPending counts the boxes
// that exist anywhere; each warp keeps its own running change (children made minus boxes
// bound) and adds it in before every push to the ring and whenever it runs out of work, so
// the counter stays at or above the true count and reaches 0 only at the end.
template <int K>
__global__ void __launch_bounds__(kBlock) k_sub_queue(SubArgs a)
{
    constexpr int N = 2 * K;
    __shared__ uint64_t stacks[kBlock / 32][kLocal];
    const Af<N + 1> em1 = em1_form<N + 1>(a.em1[0], a.em1[1]);
    const int lane = (int)(threadIdx.x & 31);
    const uint32_t lt = (1u << lane) - 1u;
    uint64_t* stk = stacks[threadIdx.x >> 5];
    const uint64_t cap = a.ringCapacity;
    volatile uint64_t* ring = a.ring;
    const unsigned long long lowWater = (unsigned long long)gridDim.x * (kBlock / 32) * 32;
    int top = 0;              // boxes on the warp's stack (warp-uniform)
    long long delta = 0;      // boxes made minus boxes bound since the last add-in (warp-uniform)
    uint64_t claim = kNoClaim;
    uint32_t tested = 0, culled = 0, idle = 0, sleep = 64, passes = 0;
    bool failed = false;
    for (;;) {
        uint64_t ent = 0;
        bool have = false;
        // (1) a claimed ring slot whose entry has been stored
        if (claim != kNoClaim) {
            const uint64_t slot = claim % cap;
            const uint64_t v = ring[slot];
            if ((v & (kQueued | kLapMask)) == queued_entry(0ull, claim, cap)) {
                ring[slot] = 0ull;
                ent = v & ~(kQueued | kLapMask);
                have = true;
                claim = kNoClaim;
            }
        }
        // (2) free lanes take the newest boxes of the warp's stack
        const uint32_t free1 = __ballot_sync(0xFFFFFFFFu, !have && claim == kNoClaim);
        const int take = min(__popc(free1), top);
        if ((free1 >> lane) & 1u) {
            const int r = __popc(free1 & lt);
            if (r < take) {
                ent = stk[top - 1 - r];
                have = true;
            }
        }
        top -= take;
        __syncwarp();
        // (3) with the stack empty, lanes still free claim ring entries
        const uint32_t free2 = __ballot_sync(0xFFFFFFFFu, !have && claim == kNoClaim);
        if (top == 0 && free2) {
            unsigned long long h = 0;
            int c = 0;
            if (lane == 0) {
                const unsigned long long t = ld_volatile(a.qTail), h0 = ld_volatile(a.qHead);
                if (h0 < t) {
                    c = (int)min((unsigned long long)__popc(free2), t - h0);
                    h = atomicAdd(a.qHead, (unsigned long long)c);
                }
            }
            c = __shfl_sync(0xFFFFFFFFu, c, 0);
            h = __shfl_sync(0xFFFFFFFFu, h, 0);
            if ((free2 >> lane) & 1u) {
                const int r = __popc(free2 & lt);
                if (r < c) claim = h + (uint64_t)r;
            }
        }
        const uint32_t work = __ballot_sync(0xFFFFFFFFu, have);
        if (!work) {
            if (top == 0) {
                // out of work: add the running change in; stop once no box is left anywhere
                // (then no entry will ever be stored in a slot still claimed here: such a
                // claim ran ahead of the producers)
                if (delta != 0) {
                    if (lane == 0) atomicAdd(a.qPending, (unsigned long long)delta);
                    delta = 0;
                }
                int done = 0;
                if (lane == 0) done = ld_volatile(a.qPending) == 0 ? 1 : 0;
                if (__shfl_sync(0xFFFFFFFFu, done, 0)) break;
            }
            if (++idle >= kQueueSpin) {
                failed = true;
                break;
            }
            __nanosleep(sleep);
            sleep = min(sleep * 2, 2048u);
            continue;
        }
        idle = 0;
        sleep = 64;
        // (4) bound the boxes
        int v = kCull;
        uint32_t row = 0, path = 0;
        int depth = 0;
        if (have) {
            row = (uint32_t)(ent >> 32);
            path = (uint32_t)ent & kPathMask;
            depth = (int)(((uint32_t)ent >> kMaxDepth) & 31u);
            Chain<K> ch;
            uint32_t q;
            load_row<K>(ch, a, row, &q);
            float lo[N], hi[N];
            box_bounds<N>(path, depth, lo, hi);
            v = bound_box<K>(ch, a.pBeg, a.pEnd[q], a.events, em1, lo, hi, a.eps);
            if (v == kSplit && depth >= a.maxDepth) v = kLeaf;
            tested++;
            culled += v == kCull;
        }
        const unsigned long long ls = warp_append(a.nLeaves, have && v == kLeaf);
        if (have && v == kLeaf) {
            if (ls < a.capacity) a.leaves[ls] = make_entry(row, depth, path);
            else raise_error(a.status, kErrCapacity);
        }
        // (5) children onto the warp's stack while it has room, the rest to the ring
        const bool split = have && v == kSplit;
        const uint32_t splits = __ballot_sync(0xFFFFFFFFu, split);
        const int made = 2 * __popc(splits);
        delta += made - __popc(work);
        const int room = kLocal - top;
        const int r2 = 2 * __popc(splits & lt);
        const uint64_t e0 = make_entry(row, depth + 1, path);
        const uint64_t e1 = make_entry(row, depth + 1, path | (1u << depth));
        bool out0 = false, out1 = false;
        if (split) {
            if (r2 < room) stk[top + r2] = e0;
            else out0 = true;
            if (r2 + 1 < room) stk[top + r2 + 1] = e1;
            else out1 = true;
        }
        top += min(made, room);
        __syncwarp();
        if (__any_sync(0xFFFFFFFFu, out0 || out1)) {
            if (lane == 0) atomicAdd(a.qPending, (unsigned long long)delta);
            delta = 0;
            if (!ring_push(a, out0, e0) || !ring_push(a, out1, e1)) {
                failed = true;
                break;
            }
        }
        // (6) lend the oldest boxes (the shallowest: the most work) when the ring runs low
        if (top > kDonateAbove && (kLendEvery == 1 || (++passes % kLendEvery) == 0)) {
            int lend = 0;
            if (lane == 0) {
                const unsigned long long t = ld_volatile(a.qTail), h0 = ld_volatile(a.qHead);
                lend = t < h0 + lowWater ? min(32, top / 2) : 0;
            }
            lend = __shfl_sync(0xFFFFFFFFu, lend, 0);
            if (lend > 0) {
                if (lane == 0) atomicAdd(a.qPending, (unsigned long long)delta);
                delta = 0;
                const uint64_t mine = lane < lend ? stk[lane] : 0ull;
                __syncwarp();
                for (int b = 0; b < top - lend; b += 32) {
                    const int i = b + lane;
                    const uint64_t x = i < top - lend ? stk[lend + i] : 0ull;
                    __syncwarp();
                    if (i < top - lend) stk[i] = x;
                    __syncwarp();
                }
                top -= lend;
                if (!ring_push(a, lane < lend, mine)) {
                    failed = true;
                    break;
                }
            }
        }
    }
    if (failed && lane == 0) raise_error(a.status, kErrSpinLimit);
    if (a.stats) {
        warp_sum(a.stats + kStTested, tested);
        warp_sum(a.stats + kStCulled, culled);
    }
}

// FP64 polish of a float root (4 Newton steps); kept when it converged next to the root.
template <int K>
__device__ __noinline__ void polish_root(float* xs, const Chain<K>& ch, float3 pBeg, float3 pEnd, uint32_t events,
                                         float eta)
{
    double xd[2 * K];
#pragma unroll
    for (int i = 0; i < 2 * K; i++) xd[i] = xs[i];
    const bool ok = solver::solve_constraints<double, K>(xd, solver::v3f<double>(pBeg), solver::v3f<double>(pEnd), ch,
                                                         (double)eta, events, 4, 1.0e-24, 4);
    double moved = 0.0;
#pragma unroll
    for (int i = 0; i < 2 * K; i++) moved = fmax(moved, fabs(xd[i] - (double)xs[i]));
    if (ok && moved < 1.0e-3) {
#pragma unroll
        for (int i = 0; i < 2 * K; i++) xs[i] = (float)xd[i];
    }
}

// One thread per leaf: the box's residual forms once, then for every bin the test of
// bin_may_hold_root; the (leaf, bin) pairs that pass go to the solve list (leaf << 8 | bin).
template <int K>
__global__ void __launch_bounds__(kBlock) k_sub_leaf_test(SubArgs a)
{
    constexpr int N = 2 * K;
    __shared__ float2 binSymbol[kMaxBins];
    const uint64_t nLeaves = min((uint64_t)*a.nLeaves, a.capacity);
    const Af<N + 1> em1 = em1_form<N + 1>(a.em1[0], a.em1[1]);
    for (uint32_t b = threadIdx.x; b < a.nBins; b += blockDim.x) {
        const float e = a.etas[b];
        float lo, hi;
        bin_symbol(em1, __fsub_rn(__fmul_rn(e, e), 1.0f), &lo, &hi);
        binSymbol[b] = make_float2(lo, hi);
    }
    __syncthreads();
    uint32_t excluded = 0;
    for (uint64_t li = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; li < nLeaves;
         li += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t ent = a.leaves[li];
        const uint32_t row = (uint32_t)(ent >> 32), path = (uint32_t)ent & kPathMask;
        const int depth = (int)(((uint32_t)ent >> kMaxDepth) & 31u);
        Chain<K> ch;
        uint32_t q;
        load_row<K>(ch, a, row, &q);
        float lo[N], hi[N];
        box_bounds<N>(path, depth, lo, hi);
        VertexForms forms[K];
        LinearRows<K> rows;
        const bool live = bound_box<K>(ch, a.pBeg, a.pEnd[q], a.events, em1, lo, hi, a.eps, forms, &rows) != kCull;
        if (a.nBins <= 64) {
            // the passing bins as a mask, then one warp-wide append for all of them
            uint64_t mask = 0;
            for (uint32_t b = 0; b < a.nBins; b++) {
                const float2 sym = binSymbol[b];
                if (live && bin_may_hold_root<K>(forms, sym.x, sym.y) && !bin_linear_excludes<K>(rows, sym.x, sym.y))
                    mask |= 1ull << b;
            }
            const uint32_t cnt = (uint32_t)__popcll(mask);
            excluded += a.nBins - cnt;
            unsigned long long slot = warp_reserve(a.nItems, cnt);
            for (; mask; mask &= mask - 1, slot++) {
                if (slot < a.itemCapacity) a.items[slot] = (li << 8) | (uint64_t)__ffsll((long long)mask) - 1;
                else raise_error(a.status, kErrCapacity);
            }
        } else {
            for (uint32_t b = 0; b < a.nBins; b++) {
                const float2 sym = binSymbol[b];
                const bool pass = live && bin_may_hold_root<K>(forms, sym.x, sym.y) &&
                                  !bin_linear_excludes<K>(rows, sym.x, sym.y);
                excluded += !pass;
                const unsigned long long s = warp_append(a.nItems, pass);
                if (pass) {
                    if (s < a.itemCapacity) a.items[s] = (li << 8) | b;
                    else raise_error(a.status, kErrCapacity);
                }
            }
        }
    }
    if (a.stats) warp_sum(a.stats + kStExcluded, excluded);
}

// One thread per (leaf, bin) pair of the solve list: Newton from the box centre,
// ownership, throughput, root output.
template <int K, bool kPolish>
__global__ void __launch_bounds__(kBlock) k_sub_leaf_solve(SubArgs a)
{
    constexpr int N = 2 * K;
    const uint64_t nItems = min((uint64_t)*a.nItems, a.itemCapacity);
    const uint32_t root = __ldg(a.root);
    uint32_t nSolves = 0, nConverged = 0, nOutside = 0, nRoots = 0;
    for (uint64_t it = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; it < nItems;
         it += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t item = a.items[it];
        const uint64_t ent = a.leaves[item >> 8];
        const uint32_t bin = (uint32_t)(item & 0xFFu);
        const uint32_t row = (uint32_t)(ent >> 32), path = (uint32_t)ent & kPathMask;
        const int depth = (int)(((uint32_t)ent >> kMaxDepth) & 31u);
        Chain<K> ch;
        uint32_t q;
        load_row<K>(ch, a, row, &q);
        float lo[N], hi[N], xs[N];
        box_bounds<N>(path, depth, lo, hi);
#pragma unroll
        for (int j = 0; j < N; j++) xs[j] = __fmul_rn(__fadd_rn(lo[j], hi[j]), 0.5f);
        const float eta = a.etas[bin];
        const float3 pEnd = a.pEnd[q];
        const bool conv = solver::solve_constraints<float, K>(xs, solver::v3f<float>(a.pBeg), solver::v3f<float>(pEnd),
                                                              ch, eta, a.events, a.maxIterations, a.costTolerance,
                                                              a.warmUp);
        bool inside = conv;
#pragma unroll
        for (int j = 0; j < N; j++)
            inside = inside && lo[j] <= xs[j] && (xs[j] < hi[j] || (hi[j] == 1.0f && xs[j] == 1.0f));
        if (kPolish && inside) polish_root<K>(xs, ch, a.pBeg, pEnd, a.events, eta);
        float thr = 0.0f;
        if (inside)
            thr = solver::contributable_throughput<float, K>(xs, solver::v3f<float>(a.pBeg), solver::v3f<float>(pEnd),
                                                             ch, a.events, a.nodes, a.sceneTris, root, eta);
        const bool emit = thr > 0.0f;
        nSolves++;
        nConverged += conv;
        nOutside += conv && !inside;
        nRoots += emit;
        const unsigned long long s = warp_append(a.nRoots, emit);
        if (emit) {
            if (s < a.rootCapacity) {
                pz_specular_root o;
                o.tuple = row;
                o.bin = bin;
                o.depth = (uint32_t)depth;
                o.path = path;
#pragma unroll
                for (int j = 0; j < 8; j++) o.params[j] = j < N ? xs[j] : 0.0f;
                o.throughput = thr;
                o.pad[0] = o.pad[1] = o.pad[2] = 0;
                a.roots[s] = o;
            } else {
                raise_error(a.status, kErrCapacity);
            }
        }
    }
    if (a.stats) {
        warp_sum(a.stats + kStSolves, nSolves);
        warp_sum(a.stats + kStConverged, nConverged);
        warp_sum(a.stats + kStOutside, nOutside);
        warp_sum(a.stats + kStRoots, nRoots);
        if (kPolish) warp_sum(a.stats + kStPolished, nConverged - nOutside);
    }
}

// Contribution of every root to the binned spectral image: the tail of the reference's
// per-path solve (solveSpecularPath<K>, main_gpu.cu:466-486) with the wavelength fixed to
// the root's bin: throughput * I / dAdw * cos at the receiver, clamped, added to
// spectral[q][bin].  The rows' query index q is the pixel of first_diffuse.
struct ContribArgs {
    uint32_t events;
    float3 pBeg;
    float lightIntensity, radianceClamp;
    const uint32_t* tuples;
    const pz_specular_root* roots;
    uint64_t nRoots;
    const FirstDiffuse* fds;
    const float* etas;
    uint32_t nBins;
    const Tri* tris;
    const Attrib* attribs;
    float* spectral;
};

template <int K>
__global__ void __launch_bounds__(kBlock) k_sub_contribute(ContribArgs a)
{
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.nRoots;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const pz_specular_root r = a.roots[i];
        const uint32_t* t = a.tuples + (size_t)r.tuple * (1 + K);
        const uint32_t px = __ldg(t);
        int idx[K];
#pragma unroll
        for (int k = 0; k < K; k++) idx[k] = (int)__ldg(t + 1 + k);
        Chain<K> ch;
        solver::load_chain<K>(ch, a.tris, a.attribs, idx);
        float xs[2 * K];
#pragma unroll
        for (int j = 0; j < 2 * K; j++) xs[j] = r.params[j];
        const FirstDiffuse fd = a.fds[px];
        const float eta = a.etas[r.bin];
        const V3<float> L = solver::v3f<float>(a.pBeg), p = solver::v3f<float>(fd.p);
        const V3<float> v0 = solver::vertex<float, K>(ch, xs, 0);
        const float dAdwValue = solver::dadw<float, K>(L, v0 - L, p, ch, a.events, eta);
        const V3<float> vl = solver::vertex<float, K>(ch, xs, K - 1);
        const float cosv = fmaxf(solver::vdot(solver::vnormalize(vl - p), solver::v3f<float>(fd.ng)), 0.0f);
        float contrib = r.throughput * a.lightIntensity / dAdwValue * cosv;
        contrib = fminf(contrib, a.radianceClamp);
        atomicAdd(a.spectral + (size_t)px * a.nBins + r.bin, contrib);
    }
}

// Sorts the leaf list by tuple row (a stable onesweep sort on the entries' upper 32 bits,
// the frontiers as ping-pong buffer and sort scratch) so that the leaf kernels see the
// rows -- and their triangles and visibility rays -- in the work list's coherent order.
// The set of roots does not depend on the order.  Reads the leaf count back (one
// synchronisation); skipped for small lists or when the frontier cannot hold the sort's
// scratch.
static cudaError_t sort_leaves(const SubArgs& a, uint64_t* fronts[2], size_t part, cudaStream_t s)
{
    unsigned long long nl = 0;
    cudaError_t e = cudaMemcpyAsync(&nl, a.nLeaves, sizeof(nl), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return e;
    nl = std::min<unsigned long long>(nl, a.capacity);
    if (nl <= 4096 || part < pz_onesweep_scratch_bytes((uint32_t)nl)) return cudaSuccess;
    const int bits = a.nRows > 1 ? 32 - __builtin_clz(a.nRows - 1) : 1;
    const int endBit = 32 + 8 * ((bits + 7) / 8);
    if (pz_onesweep_sort(a.leaves, nullptr, fronts[0], nullptr, (uint32_t)nl, 8, 32, endBit, fronts[1], part,
                         reinterpret_cast<pz_stream_t>(s)) != PZ_OK)
        return cudaErrorUnknown;
    return cudaSuccess;
}

#ifndef PZ_SUBDIV_ROUNDS
#define PZ_SUBDIV_ROUNDS 0
#endif

template <int K>
static cudaError_t run(SubArgs& a, uint64_t* fronts[2], size_t part, unsigned long long* counts, cudaStream_t s)
{
    const int grid = num_sms() * 8;
    cudaError_t e = cudaSuccess;
    if (PZ_SUBDIV_ROUNDS) {
        // one launch per depth over the whole frontier of that depth
        k_sub_init<<<(a.nRows + kBlock - 1) / kBlock, kBlock, 0, s>>>(a, fronts[0], &counts[0]);
        e = cudaGetLastError();
        int cur = 0;
        for (int d = 0; d <= a.maxDepth && e == cudaSuccess; d++) {
            e = cudaMemsetAsync(&counts[cur ^ 1], 0, sizeof(unsigned long long), s);
            if (e != cudaSuccess) break;
            k_sub_round<K><<<grid, kBlock, 0, s>>>(a, d, fronts[cur], &counts[cur], fronts[cur ^ 1], &counts[cur ^ 1]);
            e = cudaGetLastError();
            cur ^= 1;
        }
    } else {
        // one persistent launch over the box queue (the two frontier regions, contiguous)
        a.ring = fronts[0];
        a.ringCapacity = 2 * part / sizeof(uint64_t);
        e = cudaMemsetAsync(a.ring, 0, 2 * part, s);
        if (e != cudaSuccess) return e;
        k_sub_queue_init<<<(a.nRows + kBlock - 1) / kBlock, kBlock, 0, s>>>(a);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        int perSM = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, k_sub_queue<K>, kBlock, 0);
        if (e != cudaSuccess) return e;
        k_sub_queue<K><<<num_sms() * std::max(perSM, 1), kBlock, 0, s>>>(a);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) return e;
    e = sort_leaves(a, fronts, part, s);
    if (e != cudaSuccess) return e;
    k_sub_leaf_test<K><<<grid, kBlock, 0, s>>>(a);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (a.polish) k_sub_leaf_solve<K, true><<<grid * 2, kBlock, 0, s>>>(a);
    else k_sub_leaf_solve<K, false><<<grid * 2, kBlock, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace subdiv
}  // namespace pz

using namespace pz;
using namespace pz::subdiv;

static_assert(sizeof(pz_specular_root) == 64, "pz_specular_root layout");
static_assert(56 + 8 * kNumStats <= 200, "stats fit the header before the queue words");

namespace {
constexpr size_t kHeader = 256;  // status | em1[2] | counts[2] | leaf, root, item counts | stats | queue words
}

extern "C" size_t pz_subdivide_scratch_bytes(uint64_t box_capacity)
{
    return kHeader + 3 * (((size_t)box_capacity * sizeof(uint64_t) + 255) & ~(size_t)255);
}

extern "C" int pz_subdivide_solve(int K, uint32_t events, pz_float3 p_beg, const pz_float3* p_end_dev,
                                  const uint32_t* tuples_dev, uint32_t n_tuples, const float* etas_dev, int n_bins,
                                  const pz_subdiv_params* params, const pz_triangle* triangles_dev,
                                  const pz_triangle_attrib* attribs_dev, const pz_internal_node* scene_internals_dev,
                                  const pz_triangle* scene_triangles_dev, const uint32_t* scene_root_dev,
                                  pz_specular_root* roots_dev, uint64_t root_capacity, uint64_t* n_roots_out,
                                  pz_subdiv_stats* stats_out, void* scratch_dev, size_t scratch_bytes,
                                  pz_stream_t stream)
{
    if (K < 1 || K > 4) return fail(PZ_ERR_INVALID_ARGUMENT, "pz_subdivide_solve: K must be 1..4 (got %d)", K);
    if (!n_roots_out || !params)
        return fail(PZ_ERR_INVALID_ARGUMENT, "pz_subdivide_solve: n_roots_out and params are required");
    *n_roots_out = 0;
    if (stats_out) *stats_out = pz_subdiv_stats{};
    if (params->max_depth < 0 || params->max_depth > kMaxDepth)
        return fail(PZ_ERR_INVALID_ARGUMENT, "pz_subdivide_solve: max_depth must be 0..%d (got %d)", kMaxDepth,
                    params->max_depth);
    if (n_bins < 1 || n_bins > kMaxBins)
        return fail(PZ_ERR_INVALID_ARGUMENT, "pz_subdivide_solve: n_bins must be 1..%d (got %d)", kMaxBins, n_bins);
    if (!(params->eps >= 0.0f) || params->max_iterations < 1)
        return fail(PZ_ERR_INVALID_ARGUMENT, "pz_subdivide_solve: bad eps or max_iterations");
    if (n_tuples == 0) {
        clear_error();
        return PZ_OK;
    }
    if (!p_end_dev || !tuples_dev || !etas_dev || !triangles_dev || !attribs_dev || !scene_internals_dev ||
        !scene_triangles_dev || !scene_root_dev || !scratch_dev || (root_capacity > 0 && !roots_dev))
        return fail(PZ_ERR_INVALID_ARGUMENT, "pz_subdivide_solve: null buffer");
    if (reinterpret_cast<uintptr_t>(scratch_dev) & 255)
        return fail(PZ_ERR_INVALID_ARGUMENT, "pz_subdivide_solve: scratch needs 256-byte alignment");
    if (scratch_bytes < pz_subdivide_scratch_bytes(n_tuples))
        return fail(PZ_ERR_SCRATCH_TOO_SMALL, "pz_subdivide_solve: scratch %zu < %zu (a frontier must hold the tuples)",
                    scratch_bytes, pz_subdivide_scratch_bytes(n_tuples));
    const size_t part = ((scratch_bytes - kHeader) / 3) & ~(size_t)255;
    char* base = static_cast<char*>(scratch_dev);
    uint32_t* status = reinterpret_cast<uint32_t*>(base);
    float* em1 = reinterpret_cast<float*>(base + 8);
    unsigned long long* counts = reinterpret_cast<unsigned long long*>(base + 16);  // [2]
    unsigned long long* nLeaves = reinterpret_cast<unsigned long long*>(base + 32);
    unsigned long long* nRoots = reinterpret_cast<unsigned long long*>(base + 40);
    unsigned long long* nItems = reinterpret_cast<unsigned long long*>(base + 48);
    unsigned long long* stats = reinterpret_cast<unsigned long long*>(base + 56);  // [kNumStats]
    uint64_t* fronts[2] = {reinterpret_cast<uint64_t*>(base + kHeader),
                           reinterpret_cast<uint64_t*>(base + kHeader + part)};
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);

    SubArgs a;
    a.events = events;
    a.pBeg = make_float3(p_beg.x, p_beg.y, p_beg.z);
    a.pEnd = reinterpret_cast<const float3*>(p_end_dev);
    a.tuples = tuples_dev;
    a.nRows = n_tuples;
    a.etas = etas_dev;
    a.nBins = (uint32_t)n_bins;
    a.maxDepth = params->max_depth;
    a.eps = params->eps;
    a.maxIterations = params->max_iterations;
    a.costTolerance = params->cost_tolerance;
    a.warmUp = params->early_term_warmup;
    a.polish = params->fp64_polish;
    a.tris = reinterpret_cast<const Tri*>(triangles_dev);
    a.attribs = reinterpret_cast<const Attrib*>(attribs_dev);
    a.nodes = reinterpret_cast<const Node*>(scene_internals_dev);
    a.sceneTris = reinterpret_cast<const Tri*>(scene_triangles_dev);
    a.root = scene_root_dev;
    a.capacity = part / sizeof(uint64_t);
    a.em1 = em1;
    a.leaves = reinterpret_cast<uint64_t*>(base + kHeader + 2 * part);
    a.nLeaves = nLeaves;
    a.items = fronts[0];  // the frontiers are free once the rounds are done
    a.nItems = nItems;
    a.itemCapacity = 2 * a.capacity;
    a.roots = roots_dev;
    a.nRoots = nRoots;
    a.rootCapacity = root_capacity;
    a.stats = stats;
    a.status = status;
    a.qHead = reinterpret_cast<unsigned long long*>(base + 200);
    a.qTail = reinterpret_cast<unsigned long long*>(base + 208);
    a.qPending = reinterpret_cast<unsigned long long*>(base + 216);
    a.ring = nullptr;
    a.ringCapacity = 0;

    cudaError_t e = cudaMemsetAsync(base, 0, kHeader, s);
    if (e == cudaSuccess) {
        switch (K) {
            case 1: e = run<1>(a, fronts, part, counts, s); break;
            case 2: e = run<2>(a, fronts, part, counts, s); break;
            case 3: e = run<3>(a, fronts, part, counts, s); break;
            default: e = run<4>(a, fronts, part, counts, s); break;
        }
    }
    if (e != cudaSuccess) return cuda_fail(e, "pz_subdivide_solve: launch");
    unsigned long long hdr[7 + kNumStats];
    e = cudaMemcpyAsync(hdr, base, sizeof(hdr), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(e, "pz_subdivide_solve: results");
    const uint32_t st = (uint32_t)(hdr[0] & 0xFFFFFFFFull);
    *n_roots_out = hdr[5];
    if (stats_out) {
        stats_out->boxes_tested = hdr[7 + kStTested];
        stats_out->boxes_culled = hdr[7 + kStCulled];
        stats_out->leaves = hdr[4];
        stats_out->bins_excluded = hdr[7 + kStExcluded];
        stats_out->solves = hdr[7 + kStSolves];
        stats_out->converged = hdr[7 + kStConverged];
        stats_out->outside_box = hdr[7 + kStOutside];
        stats_out->roots = hdr[7 + kStRoots];
        stats_out->polished = hdr[7 + kStPolished];
    }
    if (st & kErrCapacity)
        return fail(PZ_ERR_DEVICE, "pz_subdivide_solve: capacity exceeded (%llu roots for %llu slots, or the box / solve lists)",
                    (unsigned long long)hdr[5], (unsigned long long)root_capacity);
    clear_error();
    return PZ_OK;
}

extern "C" int pz_subdivide_contribute(int K, uint32_t events, pz_float3 p_beg, float light_intensity,
                                       float radiance_clamp, const uint32_t* tuples_dev,
                                       const pz_specular_root* roots_dev, uint64_t n_roots,
                                       const void* first_diffuse_dev, const float* etas_dev, int n_bins,
                                       const pz_triangle* triangles_dev, const pz_triangle_attrib* attribs_dev,
                                       float* spectral_dev, pz_stream_t stream)
{
    if (K < 1 || K > 4) return fail(PZ_ERR_INVALID_ARGUMENT, "pz_subdivide_contribute: K must be 1..4 (got %d)", K);
    if (n_bins < 1 || n_bins > kMaxBins)
        return fail(PZ_ERR_INVALID_ARGUMENT, "pz_subdivide_contribute: n_bins must be 1..%d", kMaxBins);
    if (n_roots == 0) {
        clear_error();
        return PZ_OK;
    }
    if (!tuples_dev || !roots_dev || !first_diffuse_dev || !etas_dev || !triangles_dev || !attribs_dev ||
        !spectral_dev)
        return fail(PZ_ERR_INVALID_ARGUMENT, "pz_subdivide_contribute: null buffer");
    ContribArgs a;
    a.events = events;
    a.pBeg = make_float3(p_beg.x, p_beg.y, p_beg.z);
    a.lightIntensity = light_intensity;
    a.radianceClamp = radiance_clamp;
    a.tuples = tuples_dev;
    a.roots = roots_dev;
    a.nRoots = n_roots;
    a.fds = static_cast<const FirstDiffuse*>(first_diffuse_dev);
    a.etas = etas_dev;
    a.nBins = (uint32_t)n_bins;
    a.tris = reinterpret_cast<const Tri*>(triangles_dev);
    a.attribs = reinterpret_cast<const Attrib*>(attribs_dev);
    a.spectral = spectral_dev;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const unsigned grid = (unsigned)std::min<uint64_t>((n_roots + kBlock - 1) / kBlock, (uint64_t)num_sms() * 16);
    switch (K) {
        case 1: k_sub_contribute<1><<<grid, kBlock, 0, s>>>(a); break;
        case 2: k_sub_contribute<2><<<grid, kBlock, 0, s>>>(a); break;
        case 3: k_sub_contribute<3><<<grid, kBlock, 0, s>>>(a); break;
        default: k_sub_contribute<4><<<grid, kBlock, 0, s>>>(a); break;
    }
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "pz_subdivide_contribute");
    clear_error();
    return PZ_OK;
}
