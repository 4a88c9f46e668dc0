// pz_oracle_subdiv.hpp -- TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of the per-tuple parametric-domain subdivision solve
// (palzilla_b200/csrc/pz_subdiv.cu, C ABI pz_subdivide_solve), the parity checker for
// that kernel.  The reference has no counterpart: it solves each admissible tuple once
// from one start (main.cpp:1052).  What this file restates:
//   - the domain of a tuple row {q, tri[0..K)} is the unit box of its 2K barycentrics;
//     split t halves dimension t mod 2K; a box is (depth, path bits);
//   - a box is dropped when it lies outside a triangle, when the cosines at a vertex rule
//     the event out (the test of contributableThroughput, pk.h:760-842), when an affine
//     bound of the residual of solveConstraints<K> (pk.h:466-592; cross product of the
//     outgoing direction with the reflected / refracted one) excludes zero, or when the
//     joint linear test of two residual components per vertex excludes a root;
//   - eta^2 - 1 over the bins is one more noise symbol of the bound;
//   - a box stops splitting at max_depth or when every bounded residual component is
//     narrower than eps; at such a leaf every bin's value of eta^2 - 1 is substituted
//     into the residual forms and the joint linear test, and for the bins that pass both
//     the box centre starts the Newton solve (solve_constraints in pz_oracle.hpp); a root
//     is kept when it converged, lies in the box (half-open) and its contributable
//     throughput is positive.
// Affine arithmetic: central and linear coefficients round to nearest, every rounding
// error and nonlinear remainder is added to the radius rounded upward.
//
// Directed rounding is computed exactly from round-to-nearest results, without changing
// the FPU's rounding mode:
//   - sums: the error of s = a + b is exact (Knuth's TwoSum); the upward result is the
//     next float above s when that error is positive;
//   - products: a * b of two floats is exact in double (48 significant bits), and is
//     compared with its float rounding;
//   - quotients and square roots: the residual a - q b (resp. a - s s) is exact in
//     double and gives the side of the exact value.
// These are the IEEE directed results that the GPU's __fadd_ru, __fmul_rd, __fdiv_rd,
// __fsqrt_ru ... intrinsics return, so the box decisions equal the kernel's bit for bit.
#pragma once

#include <cmath>
#include <cstdint>
#include <vector>

namespace pzo {
namespace subdiv {

inline float up(float x) { return std::nextafter(x, INFINITY); }
inline float dn(float x) { return std::nextafter(x, -INFINITY); }
// exact error of the round-to-nearest sum s = a + b
inline float two_sum_err(float a, float b, float s)
{
    const float bb = s - a;
    return (a - (s - bb)) + (b - bb);
}
inline float add_u(float a, float b) { const float s = a + b; return two_sum_err(a, b, s) > 0.0f ? up(s) : s; }
inline float add_d(float a, float b) { const float s = a + b; return two_sum_err(a, b, s) < 0.0f ? dn(s) : s; }
inline float sub_u(float a, float b) { return add_u(a, -b); }
inline float sub_d(float a, float b) { return add_d(a, -b); }
inline float mul_u(float a, float b)
{
    const double p = (double)a * (double)b;
    const float r = (float)p;
    return (double)r < p ? up(r) : r;
}
inline float mul_d(float a, float b)
{
    const double p = (double)a * (double)b;
    const float r = (float)p;
    return (double)r > p ? dn(r) : r;
}
inline float div_d(float a, float b)
{
    const float q = a / b;
    const double rem = std::fma(-(double)q, (double)b, (double)a);  // a - q b, exact
    return (rem < 0.0) != (b < 0.0) && rem != 0.0 ? dn(q) : q;
}
inline float div_u(float a, float b)
{
    const float q = a / b;
    const double rem = std::fma(-(double)q, (double)b, (double)a);
    return (rem > 0.0) == (b > 0.0) && rem != 0.0 ? up(q) : q;
}
inline float sqrt_u(float a)
{
    const float s = std::sqrt(a);
    return (double)a - (double)s * (double)s > 0.0 ? up(s) : s;
}
inline float sqrt_d(float a)
{
    const float s = std::sqrt(a);
    return (double)a - (double)s * (double)s < 0.0 ? dn(s) : s;
}

// bound on the rounding error of one round-to-nearest result
inline float rerr(float r) { return add_u(mul_u(std::fabs(r), 0x1p-24f), 0x1p-149f); }

template <int N> struct Af { float c; float x[N]; float r; };
template <int N> struct Af3 { Af<N> x, y, z; };

template <int N> Af<N> cst(float v) { Af<N> o{}; o.c = v; return o; }

template <int N> Af<N> add(const Af<N>& a, const Af<N>& b)
{
    Af<N> o;
    o.c = a.c + b.c;
    float r = add_u(add_u(a.r, b.r), rerr(o.c));
    for (int i = 0; i < N; i++) { o.x[i] = a.x[i] + b.x[i]; r = add_u(r, rerr(o.x[i])); }
    o.r = r;
    return o;
}
template <int N> Af<N> sub(const Af<N>& a, const Af<N>& b)
{
    Af<N> o;
    o.c = a.c - b.c;
    float r = add_u(add_u(a.r, b.r), rerr(o.c));
    for (int i = 0; i < N; i++) { o.x[i] = a.x[i] - b.x[i]; r = add_u(r, rerr(o.x[i])); }
    o.r = r;
    return o;
}
template <int N> Af<N> neg(const Af<N>& a)
{
    Af<N> o;
    o.c = -a.c;
    for (int i = 0; i < N; i++) o.x[i] = -a.x[i];
    o.r = a.r;
    return o;
}
template <int N> float rad(const Af<N>& a)
{
    float s = a.r;
    for (int i = 0; i < N; i++) s = add_u(s, std::fabs(a.x[i]));
    return s;
}
template <int N> float lo(const Af<N>& a) { return sub_d(a.c, rad(a)); }
template <int N> float hi(const Af<N>& a) { return add_u(a.c, rad(a)); }
template <int N> Af<N> mul(const Af<N>& a, const Af<N>& b)
{
    Af<N> o;
    o.c = a.c * b.c;
    float r = rerr(o.c);
    float ra = a.r, rb = b.r;
    for (int i = 0; i < N; i++) {
        const float p = a.c * b.x[i], q = b.c * a.x[i];
        o.x[i] = p + q;
        r = add_u(r, add_u(add_u(rerr(p), rerr(q)), rerr(o.x[i])));
        ra = add_u(ra, std::fabs(a.x[i]));
        rb = add_u(rb, std::fabs(b.x[i]));
    }
    r = add_u(r, mul_u(std::fabs(a.c), b.r));
    r = add_u(r, mul_u(std::fabs(b.c), a.r));
    o.r = add_u(r, mul_u(ra, rb));
    return o;
}
template <int N> Af<N> scale(const Af<N>& a, float s)
{
    Af<N> o;
    o.c = a.c * s;
    float r = add_u(mul_u(a.r, std::fabs(s)), rerr(o.c));
    for (int i = 0; i < N; i++) { o.x[i] = a.x[i] * s; r = add_u(r, rerr(o.x[i])); }
    o.r = r;
    return o;
}
template <int N> Af<N> addc(const Af<N>& a, float s)
{
    Af<N> o = a;
    o.c = a.c + s;
    o.r = add_u(a.r, rerr(o.c));
    return o;
}
// min-range linearisation of sqrt on [lo, hi]
template <int N> Af<N> sqrt_af(const Af<N>& a)
{
    const float l = std::fmax(lo(a), 0.0f), h = hi(a);
    if (!(h > 0.0f)) return cst<N>(0.0f);
    const float sh = sqrt_u(h);
    const float alpha = div_d(1.0f, mul_u(2.0f, sh));
    const float dlo = sub_d(sqrt_d(l), mul_u(alpha, l));
    const float dhi = sub_u(sh, mul_d(alpha, h));
    const float zeta = (dlo + dhi) * 0.5f;
    const float delta = std::fmax(sub_u(dhi, zeta), sub_u(zeta, dlo));
    Af<N> o = addc(scale(a, alpha), zeta);
    o.r = add_u(o.r, delta);
    return o;
}
template <int N> Af3<N> sub3(const Af3<N>& a, const Af3<N>& b) { return {sub(a.x, b.x), sub(a.y, b.y), sub(a.z, b.z)}; }
template <int N> Af3<N> add3(const Af3<N>& a, const Af3<N>& b) { return {add(a.x, b.x), add(a.y, b.y), add(a.z, b.z)}; }
template <int N> Af3<N> mul3(const Af3<N>& a, const Af<N>& s) { return {mul(a.x, s), mul(a.y, s), mul(a.z, s)}; }
template <int N> Af<N> dot3(const Af3<N>& a, const Af3<N>& b) { return add(add(mul(a.x, b.x), mul(a.y, b.y)), mul(a.z, b.z)); }
template <int N> Af3<N> cross3(const Af3<N>& a, const Af3<N>& b)
{
    return {sub(mul(a.y, b.z), mul(a.z, b.y)), sub(mul(a.z, b.x), mul(a.x, b.z)), sub(mul(a.x, b.y), mul(a.y, b.x))};
}
template <int N> Af<N> lin(float p0, float e0, float e1, const Af<N>& u, const Af<N>& v)
{
    return add(addc(scale(u, e0), p0), scale(v, e1));
}
template <int N> Af3<N> lin3(F3 p0, F3 e0, F3 e1, const Af<N>& u, const Af<N>& v)
{
    return {lin(p0.x, e0.x, e1.x, u, v), lin(p0.y, e0.y, e1.y, u, v), lin(p0.z, e0.z, e1.z, u, v)};
}

inline void box_bounds(int N, uint32_t path, int depth, float* l, float* h)
{
    for (int j = 0; j < N; j++) {
        float a = 0.0f, w = 1.0f;
        for (int t = j; t < depth; t += N) {
            w *= 0.5f;
            if ((path >> t) & 1u) a += w;
        }
        l[j] = a;
        h[j] = a + w;
    }
}

enum { kCull = 0, kSplit = 1, kLeaf = 2 };

// one vertex's residual over a box: per component the centre, the radius without the
// eta^2 - 1 symbol, and that symbol's coefficient
struct VertexForms {
    bool valid;
    float c[3], rad[3], xe[3];
};

// Joint linear test over the box: rows c0_j + sum_l A_jl e_l + d_j, |d_j| <= r_j,
// e in [-1, 1]^n.  A solution has e = -Y c0 - Y d + (I - Y A) e for any Y (here A's
// inverse by Gauss-Jordan with partial pivoting, rounded to nearest); true when that
// enclosure, rounded outward, misses [-1, 1] in some coordinate.
template <int n> struct LinearTest {
    bool ok;
    float Y[n][n];
    float e[n];  // sum_l |(I - Y A)_il|, rounded up
};

template <int n>
void linear_prepare(LinearTest<n>& T, const float (&A)[n][n])
{
    float M[n][2 * n];
    for (int i = 0; i < n; i++)
        for (int j = 0; j < 2 * n; j++) M[i][j] = j < n ? A[i][j] : (j - n == i ? 1.0f : 0.0f);
    T.ok = false;
    for (int col = 0; col < n; col++) {
        int piv = col;
        float best = std::fabs(M[col][col]);
        for (int i = col + 1; i < n; i++)
            if (std::fabs(M[i][col]) > best) {
                best = std::fabs(M[i][col]);
                piv = i;
            }
        for (int j = 0; j < 2 * n; j++) std::swap(M[col][j], M[piv][j]);
        if (!(std::fabs(M[col][col]) > 0.0f)) return;
        const float inv = 1.0f / M[col][col];
        for (int j = 0; j < 2 * n; j++) M[col][j] = M[col][j] * inv;
        for (int i = 0; i < n; i++) {
            if (i == col) continue;
            const float f = M[i][col];
            for (int j = 0; j < 2 * n; j++) M[i][j] = M[i][j] - f * M[col][j];
        }
    }
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) {
            if (!std::isfinite(M[i][n + j])) return;
            T.Y[i][j] = M[i][n + j];
        }
    for (int i = 0; i < n; i++) {
        float rad = 0.0f;
        for (int l = 0; l < n; l++) {
            float sLo = 0.0f, sHi = 0.0f;
            for (int j = 0; j < n; j++) {
                sLo = add_d(sLo, mul_d(T.Y[i][j], A[j][l]));
                sHi = add_u(sHi, mul_u(T.Y[i][j], A[j][l]));
            }
            const float d = i == l ? 1.0f : 0.0f;
            rad = add_u(rad, std::fmax(sub_u(sHi, d), sub_u(d, sLo)));
        }
        T.e[i] = rad;
    }
    T.ok = true;
}

template <int n>
bool linear_excludes(const LinearTest<n>& T, const float (&c0)[n], const float (&r)[n])
{
    if (!T.ok) return false;
    for (int i = 0; i < n; i++) {
        float lo = 0.0f, hi = 0.0f, rad = T.e[i];
        for (int j = 0; j < n; j++) {
            const float y = T.Y[i][j];
            lo = add_d(lo, mul_d(-y, c0[j]));
            hi = add_u(hi, mul_u(-y, c0[j]));
            rad = add_u(rad, mul_u(std::fabs(y), r[j]));
        }
        if (sub_d(lo, rad) > 1.0f || add_u(hi, rad) < -1.0f) return true;
    }
    return false;
}

// a leaf's joint-test rows, kept for the per-bin tests
template <int K> struct LinearRows {
    bool valid;
    LinearTest<2 * K> test;
    float c[2 * K], xe[2 * K], r[2 * K];
};

// the joint test for one bin: its eta symbol [elo, ehi] substituted into every row
template <int K>
bool bin_linear_excludes(const LinearRows<K>& L, float elo, float ehi)
{
    if (!L.valid) return false;
    float c0[2 * K], r[2 * K];
    for (int j = 0; j < 2 * K; j++) {
        const float pl = std::fmin(mul_d(L.xe[j], elo), mul_d(L.xe[j], ehi));
        const float ph = std::fmax(mul_u(L.xe[j], elo), mul_u(L.xe[j], ehi));
        const float cl = add_d(L.c[j], pl), ch = add_u(L.c[j], ph);
        c0[j] = (cl + ch) * 0.5f;
        r[j] = add_u(L.r[j], std::fmax(sub_u(ch, c0[j]), sub_u(c0[j], cl)));
    }
    return linear_excludes<2 * K>(L.test, c0, r);
}

// Noise symbols 0 .. 2K-1: the box's parameters; symbol 2K: eta^2 - 1 over the bins.
template <int K>
int bound_box(const Triangle* tris, const TriangleAttrib* attribs, F3 pBeg, F3 pEnd, uint32_t events, const Af<2 * K + 1>& em1,
              const float* bl, const float* bh, float eps, VertexForms* forms = nullptr, LinearRows<K>* rows = nullptr)
{
    constexpr int N = 2 * K + 1;
    for (int k = 0; k < K; k++)
        if (add_d(bl[2 * k], bl[2 * k + 1]) > 1.0f) return kCull;
    Af3<N> X[K + 2], Nrm[K];
    X[0] = {cst<N>(pBeg.x), cst<N>(pBeg.y), cst<N>(pBeg.z)};
    X[K + 1] = {cst<N>(pEnd.x), cst<N>(pEnd.y), cst<N>(pEnd.z)};
    for (int k = 0; k < K; k++) {
        Af<N> u = cst<N>((bl[2 * k] + bh[2 * k]) * 0.5f);
        Af<N> v = cst<N>((bl[2 * k + 1] + bh[2 * k + 1]) * 0.5f);
        u.x[2 * k] = (bh[2 * k] - bl[2 * k]) * 0.5f;
        v.x[2 * k + 1] = (bh[2 * k + 1] - bl[2 * k + 1]) * 0.5f;
        const F3 v0 = tris[k].vs[0], e0 = tris[k].vs[1] - tris[k].vs[0], e1 = tris[k].vs[2] - tris[k].vs[0];
        const F3 n0 = attribs[k].shadingNormals[0];
        const F3 ne0 = attribs[k].shadingNormals[1] - attribs[k].shadingNormals[0];
        const F3 ne1 = attribs[k].shadingNormals[2] - attribs[k].shadingNormals[0];
        X[k + 1] = lin3(v0, e0, e1, u, v);
        Nrm[k] = lin3(n0, ne0, ne1, u, v);
    }
    bool resolved = true, linear = true;
    float lc0[2 * K], lA[2 * K][2 * K], lr[2 * K], lxe[2 * K], lrn[2 * K];
    for (int k = 0; k < K; k++) {
        if (forms) forms[k].valid = false;
        Af3<N> wi = sub3(X[k], X[k + 1]);
        Af3<N> wo = sub3(X[k + 2], X[k + 1]);
        const Af3<N>& n = Nrm[k];
        const Af<N> s = dot3(wi, n), t = dot3(wo, n);
        const float sl = lo(s), sh = hi(s), tl = lo(t), th = hi(t);
        const bool refract = (events >> k) & 1u;
        if (refract ? ((sl > 0.0f && tl > 0.0f) || (sh < 0.0f && th < 0.0f))
                    : ((sl >= 0.0f && th <= 0.0f) || (sh <= 0.0f && tl >= 0.0f)))
            return kCull;
        if (sh < 0.0f) {
            std::swap(wi, wo);
        } else if (!(sl >= 0.0f)) {
            resolved = false;
            linear = false;
            continue;
        }
        const Af<N> NoN = dot3(n, n);
        const Af<N> WIoN = dot3(wi, n);
        Af3<N> w;
        if (refract) {
            const Af<N> WoW = dot3(wi, wi);
            const Af<N> kk = add(mul(mul(NoN, WoW), em1), mul(WIoN, WIoN));
            if (!(lo(kk) >= 0.0f)) { resolved = false; linear = false; continue; }
            const Af<N> g = sub(WIoN, sqrt_af(kk));
            w = add3(Af3<N>{neg(mul(wi.x, NoN)), neg(mul(wi.y, NoN)), neg(mul(wi.z, NoN))}, mul3(n, g));
        } else {
            if (!(lo(NoN) > 0.0f)) { resolved = false; linear = false; continue; }
            const Af<N> d2 = scale(WIoN, 2.0f);
            w = sub3(mul3(n, d2), mul3(wi, NoN));
        }
        const Af3<N> c = cross3(wo, w);
        const Af<N>* cc[3] = {&c.x, &c.y, &c.z};
        for (int j = 0; j < 3; j++) {
            const float l = lo(*cc[j]), h = hi(*cc[j]);
            if (l > 0.0f || h < 0.0f) return kCull;
            resolved = resolved && sub_u(h, l) < eps;
            if (forms) {
                float r = cc[j]->r;
                for (int i = 0; i < N - 1; i++) r = add_u(r, std::fabs(cc[j]->x[i]));
                forms[k].c[j] = cc[j]->c;
                forms[k].rad[j] = r;
                forms[k].xe[j] = cc[j]->x[N - 1];
            }
        }
        if (forms) forms[k].valid = true;
        // the two components of c off wo's largest axis, for the joint test
        const float ax = std::fabs(wo.x.c), ay = std::fabs(wo.y.c), az = std::fabs(wo.z.c);
        const int drop = (ax >= ay && ax >= az) ? 0 : (ay >= az ? 1 : 2);
        const Af<N>& ra = drop == 0 ? c.y : c.x;
        const Af<N>& rb = drop == 2 ? c.y : c.z;
        lc0[2 * k] = ra.c;
        lc0[2 * k + 1] = rb.c;
        for (int i = 0; i < N - 1; i++) {
            lA[2 * k][i] = ra.x[i];
            lA[2 * k + 1][i] = rb.x[i];
        }
        lr[2 * k] = add_u(ra.r, std::fabs(ra.x[N - 1]));
        lr[2 * k + 1] = add_u(rb.r, std::fabs(rb.x[N - 1]));
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

template <int M> Af<M> em1_form(float mLo, float mHi)
{
    Af<M> e = cst<M>((mLo + mHi) * 0.5f);
    e.x[M - 1] = std::fmax(sub_u(mHi, e.c), sub_u(e.c, mLo));
    return e;
}

// the eta symbol's value for the bin value m of eta^2 - 1, as an interval
template <int M> void bin_symbol(const Af<M>& em1, float m, float* elo, float* ehi)
{
    const float rad = em1.x[M - 1];
    *elo = *ehi = 0.0f;
    if (rad > 0.0f) {
        *elo = div_d(sub_d(m, em1.c), rad);
        *ehi = div_u(sub_u(m, em1.c), rad);
    }
}

// can a root for a bin (eta symbol in [elo, ehi]) lie in the box (the leaf test)?
template <int K>
bool bin_may_hold_root(const VertexForms* forms, float elo, float ehi)
{
    for (int k = 0; k < K; k++) {
        if (!forms[k].valid) continue;
        for (int j = 0; j < 3; j++) {
            const float xe = forms[k].xe[j];
            const float pl = std::fmin(mul_d(xe, elo), mul_d(xe, ehi));
            const float ph = std::fmax(mul_u(xe, elo), mul_u(xe, ehi));
            const float l = sub_d(add_d(forms[k].c[j], pl), forms[k].rad[j]);
            const float h = add_u(add_u(forms[k].c[j], ph), forms[k].rad[j]);
            if (l > 0.0f || h < 0.0f) return false;
        }
    }
    return true;
}

struct Root {
    uint32_t tuple, bin, depth, path;
    float params[8];
    float throughput;
    uint32_t pad[3];
};
static_assert(sizeof(Root) == 64, "Root layout");

struct Params {
    int maxDepth;
    float eps;
    int maxIterations;
    float costTolerance;
    int warmUp;
};

// stats: tested, culled, leaves, bins excluded, solves, converged, outside, roots
template <int K>
void solve_row(uint32_t row, const uint32_t* tuples, uint32_t events, F3 pBeg, const F3* pEnd, const float* etas, int nBins,
               const Params& P, const Triangle* soupTris, const TriangleAttrib* soupAttribs, const InternalNode* nodes,
               const Triangle* sceneTris, uint32_t root, std::vector<Root>& out, uint64_t* stats)
{
    constexpr int N = 2 * K;
    const uint32_t* t = tuples + (size_t)row * (1 + K);
    const uint32_t q = t[0];
    Triangle tris[K];
    TriangleAttrib attribs[K];
    for (int k = 0; k < K; k++) {
        tris[k] = soupTris[t[1 + k]];
        attribs[k] = soupAttribs[t[1 + k]];
    }
    float mLo = 0.0f, mHi = 0.0f;
    for (int b = 0; b < nBins; b++) {
        const float m = etas[b] * etas[b] - 1.0f;
        mLo = b == 0 ? m : std::fmin(mLo, m);
        mHi = b == 0 ? m : std::fmax(mHi, m);
    }
    const Af<N + 1> em1 = em1_form<N + 1>(mLo, mHi);
    std::vector<std::pair<int, uint32_t>> stack{{0, 0u}};
    while (!stack.empty()) {
        const auto [depth, path] = stack.back();
        stack.pop_back();
        float bl[N], bh[N];
        box_bounds(N, path, depth, bl, bh);
        int v = bound_box<K>(tris, attribs, pBeg, pEnd[q], events, em1, bl, bh, P.eps);
        if (v == kSplit && depth >= P.maxDepth) v = kLeaf;
        stats[0]++;
        if (v == kCull) { stats[1]++; continue; }
        if (v == kSplit) {
            stack.push_back({depth + 1, path | (1u << depth)});
            stack.push_back({depth + 1, path});
            continue;
        }
        stats[2]++;
        VertexForms forms[K];
        LinearRows<K> lrows;
        bound_box<K>(tris, attribs, pBeg, pEnd[q], events, em1, bl, bh, P.eps, forms, &lrows);
        for (int b = 0; b < nBins; b++) {
            float elo, ehi;
            bin_symbol(em1, etas[b] * etas[b] - 1.0f, &elo, &ehi);
            if (!bin_may_hold_root<K>(forms, elo, ehi) || bin_linear_excludes<K>(lrows, elo, ehi)) {
                stats[3]++;
                continue;
            }
            float xs[N];
            for (int j = 0; j < N; j++) xs[j] = (bl[j] + bh[j]) * 0.5f;
            const bool conv = solve_constraints<float, K>(xs, pBeg, pEnd[q], tris, attribs, etas[b], events,
                                                          P.maxIterations, P.costTolerance, P.warmUp);
            stats[4]++;
            if (!conv) continue;
            stats[5]++;
            bool inside = true;
            for (int j = 0; j < N; j++)
                inside = inside && bl[j] <= xs[j] && (xs[j] < bh[j] || (bh[j] == 1.0f && xs[j] == 1.0f));
            if (!inside) { stats[6]++; continue; }
            const float thr = contributable_throughput<float, K>(xs, pBeg, pEnd[q], tris, attribs, events, nodes,
                                                                sceneTris, root, etas[b]);
            if (!(thr > 0.0f)) continue;
            stats[7]++;
            Root r{};
            r.tuple = row;
            r.bin = (uint32_t)b;
            r.depth = (uint32_t)depth;
            r.path = path;
            for (int j = 0; j < N; j++) r.params[j] = xs[j];
            r.throughput = thr;
            out.push_back(r);
        }
    }
}

}  // namespace subdiv
}  // namespace pzo
