// pz_adjoint.cu -- the adjoint of the binned caustic render: gradients of a loss on the
// spectral image with respect to the heights (y) of the scene's vertices and to the
// Cauchy coefficients of the index of refraction.  No reference counterpart.
//
// Forward (pz_adjoint_forward): the plain binned solve in the reference's arithmetic.
// Backward (pz_adjoint_backward), one thread per (work item, bin):
//  * the path's root x* is recomputed from the photon's barycentrics (the same solve and
//    the same accept / reject decision as the forward), nothing is stored between passes;
//  * for an accepted, unclamped path the constraint C(x, p) and the contribution
//    c(x, p) = T_fresnel / dAdw * cos * I are evaluated once more with forward-mode
//    tangents for the 2K barycentrics, the 3K vertex heights of the chain's triangles and
//    eta (dAdw's own ray differentials nest inside, as dual numbers over that type);
//  * implicit-function theorem at the root: dx*/dp = -J_x^+ J_p (Householder least
//    squares on the 3K x 2K Jacobian), so dc/dp = dc/dp|_x + dc/dx dx*/dp;
//  * the loss weight dL/dI of the path's (pixel, bin) scales it; heights accumulate by
//    atomics through the triangle-corner -> vertex map, eta into dL/dA and dL/dB of
//    eta = A + B / lambda^2 (d eta / dB = (eta - A) / B).
// Visibility, the edge tests and the clamp are piecewise constant: they select paths but
// carry no gradient.
#include "pz_capi_internal.h"
#include "pz_frame.cuh"
#include "pz_solve.cuh"
#include "pz_solver.cuh"

namespace pz {
namespace adjoint {

using solver::D;
using solver::D3;
using solver::V3;
using pz::operator+;
using pz::operator-;
using pz::operator*;
using pz::operator/;

// ---------------------------------------------------------------- forward-mode scalar
template <int N> struct G {
    float v;
    float d[N];
    PZ_HD G() = default;
    PZ_HD G(float x) : v(x)
    {
#pragma unroll
        for (int i = 0; i < N; i++) d[i] = 0.0f;
    }
    PZ_HD explicit operator float() const { return v; }
};
template <int N> PZ_D G<N> operator+(const G<N>& a, const G<N>& b)
{
    G<N> r;
    r.v = a.v + b.v;
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = a.d[i] + b.d[i];
    return r;
}
template <int N> PZ_D G<N> operator-(const G<N>& a, const G<N>& b)
{
    G<N> r;
    r.v = a.v - b.v;
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = a.d[i] - b.d[i];
    return r;
}
template <int N> PZ_D G<N> operator-(const G<N>& a)
{
    G<N> r;
    r.v = -a.v;
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = -a.d[i];
    return r;
}
template <int N> PZ_D G<N> operator*(const G<N>& a, const G<N>& b)
{
    G<N> r;
    r.v = a.v * b.v;
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
    return r;
}
template <int N> PZ_D G<N> operator/(const G<N>& a, const G<N>& b)
{
    G<N> r;
    const float inv = 1.0f / b.v;
    r.v = a.v * inv;
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = (a.d[i] - r.v * b.d[i]) * inv;
    return r;
}
template <int N> PZ_D G<N>& operator+=(G<N>& a, const G<N>& b) { return a = a + b; }
template <int N> PZ_D G<N>& operator-=(G<N>& a, const G<N>& b) { return a = a - b; }
template <int N> PZ_D G<N>& operator*=(G<N>& a, const G<N>& b) { return a = a * b; }
template <int N> PZ_D bool operator<(const G<N>& a, const G<N>& b) { return a.v < b.v; }
template <int N> PZ_D bool operator>(const G<N>& a, const G<N>& b) { return a.v > b.v; }
template <int N> PZ_D bool operator==(const G<N>& a, const G<N>& b) { return a.v == b.v; }
template <int N> PZ_D bool operator!=(const G<N>& a, const G<N>& b) { return a.v != b.v; }
template <int N> PZ_D G<N> sqrt(const G<N>& a)
{
    G<N> r;
    r.v = sqrtf(a.v);
    const float h = 0.5f / r.v;
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = a.d[i] * h;
    return r;
}
template <int N> PZ_D G<N> copysign(const G<N>& a, const G<N>& b)
{
    return (signbit(a.v) != signbit(b.v)) ? -a : a;
}
template <int N> PZ_D G<N> fmaxg(const G<N>& a, const G<N>& b) { return a.v > b.v ? a : (b.v != b.v ? a : b); }
template <int N> PZ_D G<N> seed(float v, int i)
{
    G<N> r(v);
    r.d[i] = 1.0f;
    return r;
}

// ---------------------------------------------------------------- generic chain
// Triangle geometry carries the scalar type (its vertex heights are parameters); the
// shading normals are fixed attributes.
template <int K, class S> struct GChain {
    V3<S> p0[K], e0[K], e1[K], ng[K];
    float3 n0[K], ne0[K], ne1[K];
    int32_t material[K];
};

template <class S> PZ_D V3<S> gv(float3 a) { return V3<S>{S(a.x), S(a.y), S(a.z)}; }
template <class S> PZ_D V3<S> gadd(V3<S> a, V3<S> b) { return V3<S>{a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class S> PZ_D V3<S> gsub(V3<S> a, V3<S> b) { return V3<S>{a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class S> PZ_D V3<S> gmul(V3<S> a, S s) { return V3<S>{a.x * s, a.y * s, a.z * s}; }
template <class S> PZ_D V3<S> gneg(V3<S> a) { return V3<S>{-a.x, -a.y, -a.z}; }
template <class S> PZ_D S gdot(V3<S> a, V3<S> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class S> PZ_D V3<S> gcross(V3<S> a, V3<S> b)
{
    return V3<S>{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class S> PZ_D V3<S> gnormalize(V3<S> a) { return gmul(a, S(1.0f) / sqrt(gdot(a, a))); }

template <int K, class S>
PZ_D V3<S> gvertex(const GChain<K, S>& c, const S* x, int k)
{
    return gadd(gadd(c.p0[k], gmul(c.e0[k], x[2 * k])), gmul(c.e1[k], x[2 * k + 1]));
}
template <int K, class S>
PZ_D V3<S> gshading(const GChain<K, S>& c, const S* x, int k)
{
    return gnormalize(gadd(gadd(gv<S>(c.n0[k]), gmul(gv<S>(c.ne0[k]), x[2 * k])), gmul(gv<S>(c.ne1[k]), x[2 * k + 1])));
}

// normalization-free refraction (saka.h:191-202) and reflection, generic scalar
template <class S> PZ_D V3<S> grefract(V3<S> wi, V3<S> n, S eta)
{
    const S NoN = gdot(n, n), WIoN = gdot(wi, n), WoW = gdot(wi, wi);
    const S k = NoN * WoW * (eta * eta - S(1.0f)) + WIoN * WIoN;
    if (k.v < 0.0f) return V3<S>{S(0.0f), S(0.0f), S(0.0f)};
    return gadd(gmul(gneg(wi), NoN), gmul(n, WIoN - sqrt(k)));
}
template <class S> PZ_D V3<S> greflect(V3<S> wi, V3<S> n)
{
    return gsub(gmul(n, gdot(wi, n) * S(2.0f) / gdot(n, n)), wi);
}

// The 3K specular constraints at x (solveConstraints' residual, pk.h:484-548).
template <int K, class S>
PZ_D void constraints(const S* x, V3<S> L, V3<S> P, const GChain<K, S>& ch, S eta, uint32_t events, S (&c)[3 * K])
{
    V3<S> v[K + 2], sn[K];
    v[0] = L;
    v[K + 1] = P;
#pragma unroll
    for (int k = 0; k < K; k++) {
        v[k + 1] = gvertex(ch, x, k);
        sn[k] = gadd(gadd(gv<S>(ch.n0[k]), gmul(gv<S>(ch.ne0[k]), x[2 * k])), gmul(gv<S>(ch.ne1[k]), x[2 * k + 1]));
    }
#pragma unroll
    for (int k = 0; k < K; k++) {
        V3<S> wi = gsub(v[k], v[k + 1]), wo = gsub(v[k + 2], v[k + 1]);
        if (gdot(wi, sn[k]).v < 0.0f) {
            const V3<S> t = wi;
            wi = wo;
            wo = t;
        }
        const V3<S> wopt = ((events >> k) & 1u) ? grefract(wi, sn[k], eta) : greflect(wi, sn[k]);
        const V3<S> cc = gcross(wo, wopt);
        c[3 * k + 0] = cc.x;
        c[3 * k + 1] = cc.y;
        c[3 * k + 2] = cc.z;
    }
}

// Fresnel transmittance (fresnel_exact_norm_free) as solver::fresnel_T, generic scalar
template <class S> PZ_D S gfresnel(V3<S> wi, V3<S> n, S eta)
{
    const S nn = gdot(n, n), wiwi = gdot(wi, wi);
    S C = gdot(n, wi);
    if (C.v < 0.0f) {
        C = -C;
        n = gneg(n);
        eta = S(1.0f) / eta;
    }
    const S K2 = nn * wiwi * (eta * eta - S(1.0f)) + C * C;
    if (K2.v < 0.0f) return S(1.0f);
    const S Gs = sqrt(K2);
    const S GmC = Gs - C, GpC = Gs + C;
    const S a = GmC / GpC, b = (C * GpC - nn * wiwi) / (C * GmC + nn * wiwi);
    return S(0.5f) * (a * a) * (S(1.0f) + b * b);
}

// dual numbers over S for dAdw's ray differentials
template <class S> struct Dl { S v, g; };
template <class S> PZ_D Dl<S> dlc(S v) { return Dl<S>{v, S(0.0f)}; }
template <class S> PZ_D Dl<S> operator+(Dl<S> a, Dl<S> b) { return {a.v + b.v, a.g + b.g}; }
template <class S> PZ_D Dl<S> operator-(Dl<S> a, Dl<S> b) { return {a.v - b.v, a.g - b.g}; }
template <class S> PZ_D Dl<S> operator-(Dl<S> a) { return {-a.v, -a.g}; }
template <class S> PZ_D Dl<S> operator*(Dl<S> a, Dl<S> b) { return {a.v * b.v, a.g * b.v + b.g * a.v}; }
template <class S> PZ_D Dl<S> operator/(Dl<S> a, Dl<S> b)
{
    return {a.v / b.v, a.g * (S(1.0f) / b.v) + b.g * (-a.v / (b.v * b.v))};
}
template <class S> PZ_D Dl<S> dlsqrt(Dl<S> a)
{
    const S s = sqrt(a.v);
    return {s, a.g * (S(0.5f) / s)};
}
template <class S> struct Dl3 { Dl<S> x, y, z; };
template <class S> PZ_D Dl3<S> dl3(V3<S> v) { return {dlc(v.x), dlc(v.y), dlc(v.z)}; }
template <class S> PZ_D Dl3<S> operator+(Dl3<S> a, Dl3<S> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class S> PZ_D Dl3<S> operator-(Dl3<S> a, Dl3<S> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class S> PZ_D Dl3<S> operator-(Dl3<S> a) { return {-a.x, -a.y, -a.z}; }
template <class S> PZ_D Dl3<S> operator*(Dl3<S> a, Dl<S> s) { return {a.x * s, a.y * s, a.z * s}; }
template <class S> PZ_D Dl<S> dldot(Dl3<S> a, Dl3<S> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class S> PZ_D Dl3<S> dlrefract(Dl3<S> wi, Dl3<S> n, S eta)
{
    const Dl<S> NoN = dldot(n, n), WIoN = dldot(wi, n), WoW = dldot(wi, wi);
    const Dl<S> k = NoN * WoW * dlc(eta * eta - S(1.0f)) + WIoN * WIoN;
    if (k.v.v < 0.0f) return dl3(V3<S>{S(0.0f), S(0.0f), S(0.0f)});
    return -wi * NoN + n * (WIoN - dlsqrt(k));
}
template <class S> PZ_D Dl3<S> dlreflect(Dl3<S> wi, Dl3<S> n)
{
    return n * dldot(wi, n) * dlc(S(2.0f)) / dldot(n, n) - wi;
}
template <class S> PZ_D Dl3<S> operator/(Dl3<S> a, Dl<S> s) { return {a.x / s, a.y / s, a.z / s}; }

// dAdw (pk.h:844-930) with the chain geometry in S
template <int K, class S>
PZ_D S gdadw(V3<S> ro, V3<S> rd, V3<S> p_end, const GChain<K, S>& ch, uint32_t events, S eta, bool* ok)
{
    rd = gnormalize(rd);
    V3<S> dAxis[2];
    *ok = true;
#pragma unroll
    for (int i = 0; i < 2; i++) {
        Dl<S> dif[2] = {dlc(S(0.0f)), dlc(S(0.0f))};
        dif[i].g = S(1.0f);
        Dl3<S> ro_j = dl3(ro);
        const S sign = copysign(S(1.0f), rd.z);  // GetOrthonormalBasis, pk.h:453-459
        const S a = S(-1.0f) / (sign + rd.z);
        const S bb = rd.x * rd.y * a;
        const V3<S> T0{S(1.0f) + sign * rd.x * rd.x * a, sign * bb, -(sign * rd.x)};
        const V3<S> T1{bb, sign + rd.y * rd.y * a, -rd.y};
        Dl3<S> rd_j = dl3(rd) + dl3(T0) * dif[0] + dl3(T1) * dif[1];
#pragma unroll
        for (int j = 0; j < K; j++) {
            const V3<S> ng = ch.ng[j];
            const V3<S> tv0 = ch.p0[j];
            const V3<S> tv1 = gadd(tv0, ch.e0[j]);
            const V3<S> tv2 = gadd(tv0, ch.e1[j]);
            const Dl<S> t = dldot(dl3(tv0) - ro_j, dl3(ng)) / dldot(dl3(ng), rd_j);
            const Dl3<S> p = ro_j + rd_j * t;
            Dl<S> v = dldot(p - dl3(tv1), dl3(gcross(ng, gsub(tv1, tv0))));
            Dl<S> w = dldot(p - dl3(tv2), dl3(gcross(ng, gsub(tv2, tv1))));
            Dl<S> u = dldot(p - dl3(tv0), dl3(gcross(ng, gsub(tv0, tv2))));
            const Dl<S> area = u + v + w;
            u = u / area;
            v = v / area;
            w = w / area;
            const V3<S> n0 = gv<S>(ch.n0[j]);
            const V3<S> n1 = gadd(n0, gv<S>(ch.ne0[j]));
            const V3<S> n2 = gadd(n0, gv<S>(ch.ne1[j]));
            const Dl3<S> n = dl3(n0) * w + dl3(n1) * u + dl3(n2) * v;
            const Dl3<S> wi = -rd_j;
            Dl3<S> wo;
            if ((events >> j) & 1u) {
                if (dldot(wi, n).v.v < 0.0f) {
                    wo = dlrefract(wi, -n, S(1.0f) / eta);
                    if (wo.x.v.v == 0.0f && wo.y.v.v == 0.0f && wo.z.v.v == 0.0f) *ok = false;
                } else {
                    wo = dlrefract(wi, n, eta);
                }
            } else {
                wo = dlreflect(wi, n);
            }
            ro_j = p;
            rd_j = wo;
        }
        const V3<S> p_last{ro_j.x.v, ro_j.y.v, ro_j.z.v};
        const Dl3<S> pn = dl3(gsub(p_last, p_end));
        const Dl<S> t = dldot(dl3(p_end) - ro_j, pn) / dldot(pn, rd_j);
        const Dl3<S> pf = ro_j + rd_j * t;
        dAxis[i] = V3<S>{pf.x.g, pf.y.g, pf.z.g};
    }
    const S len0 = sqrt(gdot(dAxis[0], dAxis[0])), len1 = sqrt(gdot(dAxis[1], dAxis[1]));
    const V3<S> c = gcross(gmul(dAxis[0], S(1.0f) / len0), gmul(dAxis[1], S(1.0f) / len1));
    const S s = sqrt(gdot(c, c));
    return len0 * len1 * fmaxg(s, S(0.01f));
}

// Contribution of an accepted path (contributableThroughput's Fresnel product, dAdw,
// receiver cosine), without the clamp.
template <int K, class S>
PZ_D S contribution(const S* x, V3<S> L, V3<S> P, float3 ngRecv, const GChain<K, S>& ch, uint32_t events, S eta,
                    float intensity, bool* ok)
{
    V3<S> v[K + 2];
    v[0] = L;
    v[K + 1] = P;
#pragma unroll
    for (int k = 0; k < K; k++) v[k + 1] = gvertex(ch, x, k);
    S thr(1.0f);
#pragma unroll
    for (int k = 0; k < K; k++) {
        const V3<S> wi = gsub(v[k], v[k + 1]), wo = gsub(v[k + 2], v[k + 1]);
        const V3<S> n = gshading(ch, x, k);
        const bool eR = 0.0f < gdot(wi, n).v * gdot(wo, n).v;
        if (ch.material[k] == kDielectric) {
            const S r = gfresnel(wi, n, eta);
            thr = thr * (eR ? r : S(1.0f) - r);
        }
    }
    const S dadw = gdadw<K, S>(L, gsub(v[1], L), P, ch, events, eta, ok);
    const S cosv = gdot(gnormalize(gsub(v[K], P)), gv<S>(ngRecv));
    if (!(cosv.v > 0.0f)) *ok = false;
    return thr * S(intensity) / dadw * cosv;
}

struct AdjArgs {
    SolveArgs s;
    const float* dLdI;        // [pixel][bin]
    const int32_t* corner;    // [triangle][3] vertex index of each corner, or -1
    float* gradHeights;
    float* gradCauchy;        // [2]: dL/dA, dL/dB
};

// The forward's decisions for one (path, bin), recomputed: Newton from the photon's
// barycentrics, admissibility and visibility, and the clamp.  True (root in x) when the
// path contributes unclamped, so that it has a gradient.
template <int K>
PZ_D bool adj_accept(const AdjArgs& a, uint64_t pathIdx, uint32_t bin, float (&x)[2 * K])
{
    const uint32_t nb = (uint32_t)a.s.nBins;
    const SpecularPath sp = a.s.paths[pathIdx];
    if (a.dLdI[(size_t)sp.pixel * nb + bin] == 0.0f) return false;
    const FirstDiffuse fd = a.s.fds[sp.pixel];
    const int4 ti = a.s.cache.tris[sp.cacheIndex];
    const int idx[4] = {ti.x, ti.y, ti.z, ti.w};
    solver::Chain<K> ch;
    solver::load_chain<K>(ch, a.s.tris, a.s.attribs, idx);
    const float4 q0 = a.s.cache.params[2 * sp.cacheIndex], q1 = a.s.cache.params[2 * sp.cacheIndex + 1];
    const float pp[8] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
#pragma unroll
    for (int i = 0; i < 2 * K; i++) x[i] = pp[i];
    const float eta = a.s.etas[bin];
    const V3<float> L = solver::v3f<float>(a.s.p_light), P = solver::v3f<float>(fd.p);
    const uint32_t root = __ldg(a.s.root);
    if (!solver::solve_constraints<float, K>(x, L, P, ch, eta, a.s.events, a.s.maxIterations, a.s.costTolerance,
                                             a.s.earlyTermWarmUp))
        return false;
    const float thr = solver::contributable_throughput<float, K>(x, L, P, ch, a.s.events, a.s.nodes, a.s.tris, root,
                                                                 eta);
    if (!(0.0f < thr)) return false;
    const V3<float> v0 = solver::vertex<float, K>(ch, x, 0);
    const float dadw = solver::dadw<float, K>(L, v0 - L, P, ch, a.s.events, eta);
    const V3<float> vl = solver::vertex<float, K>(ch, x, K - 1);
    const float cosv = fmaxf(solver::vdot(solver::vnormalize(vl - P), solver::v3f<float>(fd.ng)), 0.0f);
    const float c = thr * a.s.lightIntensity / dadw * cosv;
    return c < a.s.radianceClamp;  // clamped: no gradient
}

// The gradient of one accepted (path, bin) at its root x: implicit-function derivatives
// of the root, the contribution's forward-mode derivatives, scaled by dL/dI and added to
// the heights and the Cauchy coefficients.
template <int K>
PZ_D void adj_gradient(const AdjArgs& a, uint64_t pathIdx, uint32_t bin, const float (&x)[2 * K])
{
    constexpr int NX = 2 * K, NP = 3 * K + 1, N = NX + NP;
    using S = G<N>;
    const uint32_t nb = (uint32_t)a.s.nBins;
    const SpecularPath sp = a.s.paths[pathIdx];
    const float g = a.dLdI[(size_t)sp.pixel * nb + bin];
    const FirstDiffuse fd = a.s.fds[sp.pixel];
    const int4 ti = a.s.cache.tris[sp.cacheIndex];
    const int idx[4] = {ti.x, ti.y, ti.z, ti.w};
    solver::Chain<K> ch;
    solver::load_chain<K>(ch, a.s.tris, a.s.attribs, idx);
    const float eta = a.s.etas[bin];
    // tangent layout: [0, 2K) barycentrics, [2K, 5K) corner heights, 5K eta
    GChain<K, S> gc;
#pragma unroll
    for (int k = 0; k < K; k++) {
        V3<S> pc[3];
        float3 corners[3];
        load_tri(a.s.tris, (uint32_t)idx[k], corners[0], corners[1], corners[2]);
#pragma unroll
        for (int c = 0; c < 3; c++) {
            pc[c] = gv<S>(corners[c]);
            pc[c].y = seed<N>(corners[c].y, NX + 3 * k + c);
        }
        gc.p0[k] = pc[0];
        gc.e0[k] = gsub(pc[1], pc[0]);
        gc.e1[k] = gsub(pc[2], pc[0]);
        gc.ng[k] = gcross(gc.e0[k], gc.e1[k]);
        gc.n0[k] = ch.n0[k];
        gc.ne0[k] = ch.ne0[k];
        gc.ne1[k] = ch.ne1[k];
        gc.material[k] = ch.material[k];
    }
    S xs[NX];
#pragma unroll
    for (int i = 0; i < NX; i++) xs[i] = seed<N>(x[i], i);
    const S etaS = seed<N>(eta, NX + 3 * K);
    const V3<S> LS = gv<S>(a.s.p_light), PS = gv<S>(fd.p);
    // Jacobians of the constraints at the root
    S cst[3 * K];
    constraints<K, S>(xs, LS, PS, gc, etaS, a.s.events, cst);
    float dxdp[NP][NX];
#pragma unroll
    for (int j = 0; j < NP; j++) {
        float A[NX][3 * K], b[3 * K];
#pragma unroll
        for (int i = 0; i < NX; i++)
#pragma unroll
            for (int r = 0; r < 3 * K; r++) A[i][r] = cst[r].d[i];
#pragma unroll
        for (int r = 0; r < 3 * K; r++) b[r] = -cst[r].d[NX + j];
        solver::qr_solve<float, 3 * K, NX>(A, b, dxdp[j]);
    }
    bool ok = true;
    const S c = contribution<K, S>(xs, LS, PS, fd.ng, gc, a.s.events, etaS, a.s.lightIntensity, &ok);
    if (!ok || !(c.v == c.v)) return;
    float total[NP];
    bool finite = true;
#pragma unroll
    for (int j = 0; j < NP; j++) {
        float t = c.d[NX + j];
#pragma unroll
        for (int i = 0; i < NX; i++) t += c.d[i] * dxdp[j][i];
        total[j] = t * g;
        finite = finite && isfinite(total[j]);
    }
    if (!finite) return;  // singular Jacobian at the root: the path has no usable derivative
#pragma unroll
    for (int k = 0; k < K; k++)
#pragma unroll
        for (int cc = 0; cc < 3; cc++) {
            const int v = a.corner[3 * idx[k] + cc];
            if (v >= 0) atomicAdd(a.gradHeights + v, total[3 * k + cc]);
        }
    const float ge = total[3 * K];
    atomicAdd(a.gradCauchy + 0, ge);
    atomicAdd(a.gradCauchy + 1, ge * (eta - a.s.cauchyA) / a.s.cauchyB);
}


template <int K>
__global__ void __launch_bounds__(128) k_adjoint(AdjArgs a)
{
    const uint64_t item = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t nb = (uint32_t)a.s.nBins;
    const uint64_t pathIdx = item / nb;
    const uint32_t bin = (uint32_t)(item % nb);
    if (pathIdx >= a.s.nPaths) return;
    float x[2 * K];
    if (adj_accept<K>(a, pathIdx, bin, x)) adj_gradient<K>(a, pathIdx, bin, x);
}

// The compact form: k_adjoint_filter keeps the accepted (path, bin) pairs and their roots
// in a list (warp-aggregated appends); k_adjoint_grad differentiates only those, in full
// warps.  The filter runs the light solve code at high occupancy; the gradient's register
// footprint applies only to paths that contribute.
struct AdjRecord {
    uint32_t path, bin;
    float x[4];
    uint32_t pad[2];
};
static_assert(sizeof(AdjRecord) == 32, "AdjRecord layout");

template <int K>
__global__ void __launch_bounds__(256) k_adjoint_filter(AdjArgs a, AdjRecord* list, unsigned long long* count,
                                                        uint64_t capacity, uint32_t* status)
{
    const uint32_t nb = (uint32_t)a.s.nBins;
    const uint64_t items = a.s.nPaths * (uint64_t)nb;
    for (uint64_t item = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; item < items;
         item += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t pathIdx = item / nb;
        const uint32_t bin = (uint32_t)(item % nb);
        float x[2 * K];
        const bool keep = adj_accept<K>(a, pathIdx, bin, x);
        const uint32_t active = __activemask();
        const uint32_t ballot = __ballot_sync(active, keep);
        const int leader = __ffs(active) - 1;
        unsigned long long base = 0;
        if ((int)(threadIdx.x & 31) == leader && ballot) base = atomicAdd(count, (unsigned long long)__popc(ballot));
        base = __shfl_sync(active, base, leader);
        if (keep) {
            const unsigned long long slot = base + __popc(ballot & ((1u << (threadIdx.x & 31)) - 1u));
            if (slot < capacity) {
                AdjRecord r;
                r.path = (uint32_t)pathIdx;
                r.bin = bin;
#pragma unroll
                for (int i = 0; i < 4; i++) r.x[i] = i < 2 * K ? x[i] : 0.0f;
                r.pad[0] = r.pad[1] = 0;
                list[slot] = r;
            } else {
                raise_error(status, kErrCapacity);
            }
        }
    }
}

template <int K>
__global__ void __launch_bounds__(128) k_adjoint_grad(AdjArgs a, const AdjRecord* list,
                                                      const unsigned long long* count, uint64_t capacity)
{
    const uint64_t n = min((uint64_t)*count, capacity);
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const AdjRecord r = list[i];
        float x[2 * K];
#pragma unroll
        for (int j = 0; j < 2 * K; j++) x[j] = r.x[j];
        adj_gradient<K>(a, r.path, r.bin, x);
    }
}
}  // namespace adjoint
}  // namespace pz

using namespace pz;

namespace pz {
int solve_args_from_desc(const pz_solve_desc* desc, SolveArgs* a, const char* who);  // pz_capi_frame.cu
}

extern "C" int pz_adjoint_forward(const pz_solve_desc* desc, pz_stream_t stream)
{
    if (!desc || !desc->spectral || desc->n_bins < 1)
        return fail(PZ_ERR_INVALID_ARGUMENT, "pz_adjoint_forward: binned mode (spectral image, n_bins >= 1) required");
    SolveArgs a;
    int r = solve_args_from_desc(desc, &a, "pz_adjoint_forward");
    if (r != PZ_OK) return r;
    cudaError_t e = launch_solve_plain_exact(desc->K, true, a, reinterpret_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_fail(e, "pz_adjoint_forward");
    clear_error();
    return PZ_OK;
}

template <int K>
static cudaError_t launch_adjoint(const adjoint::AdjArgs& a, cudaStream_t s)
{
    const uint64_t items = a.s.nPaths * (uint64_t)a.s.nBins;
    if (items == 0) return cudaSuccess;
    adjoint::k_adjoint<K><<<(unsigned)((items + 127) / 128), 128, 0, s>>>(a);
    return cudaGetLastError();
}

template <int K>
static cudaError_t launch_adjoint_compact(const adjoint::AdjArgs& a, adjoint::AdjRecord* list,
                                          unsigned long long* count, uint64_t capacity, uint32_t* status,
                                          cudaStream_t s)
{
    const uint64_t items = a.s.nPaths * (uint64_t)a.s.nBins;
    if (items == 0) return cudaSuccess;
    const unsigned grid = (unsigned)std::min<uint64_t>((items + 255) / 256, (uint64_t)num_sms() * 32);
    adjoint::k_adjoint_filter<K><<<grid, 256, 0, s>>>(a, list, count, capacity, status);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    adjoint::k_adjoint_grad<K><<<num_sms() * 16, 128, 0, s>>>(a, list, count, capacity);
    return cudaGetLastError();
}

extern "C" int pz_adjoint_backward(const pz_solve_desc* desc, const float* dloss_dspectral_dev,
                                   const int32_t* corner_vertex_dev, float* grad_heights_dev, float* grad_cauchy_dev,
                                   pz_stream_t stream)
{
    if (!desc || desc->n_bins < 1 || !desc->etas)
        return fail(PZ_ERR_INVALID_ARGUMENT, "pz_adjoint_backward: binned mode (etas, n_bins >= 1) required");
    if (!dloss_dspectral_dev || !corner_vertex_dev || !grad_heights_dev || !grad_cauchy_dev)
        return fail(PZ_ERR_INVALID_ARGUMENT, "pz_adjoint_backward: null buffer");
    if (desc->cauchy_b == 0.0f) return fail(PZ_ERR_INVALID_ARGUMENT, "pz_adjoint_backward: cauchy_b must be non-zero");
    adjoint::AdjArgs a;
    int r = solve_args_from_desc(desc, &a.s, "pz_adjoint_backward");
    if (r != PZ_OK) return r;
    a.s.nBins = desc->n_bins;
    a.s.etas = desc->etas;
    a.dLdI = dloss_dspectral_dev;
    a.corner = corner_vertex_dev;
    a.gradHeights = grad_heights_dev;
    a.gradCauchy = grad_cauchy_dev;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    cudaError_t e;
    switch (desc->K) {
        case 1: e = launch_adjoint<1>(a, s); break;
        case 2: e = launch_adjoint<2>(a, s); break;
        default: return fail(PZ_ERR_UNSUPPORTED, "pz_adjoint_backward: K = %d (1 or 2 supported)", desc->K);
    }
    if (e != cudaSuccess) return cuda_fail(e, "pz_adjoint_backward");
    clear_error();
    return PZ_OK;
}

namespace {
constexpr size_t kAdjHeader = 256;  // status | record count
}

extern "C" size_t pz_adjoint_scratch_bytes(uint64_t capacity)
{
    return kAdjHeader + (size_t)capacity * sizeof(adjoint::AdjRecord);
}

extern "C" int pz_adjoint_backward_compact(const pz_solve_desc* desc, const float* dloss_dspectral_dev,
                                           const int32_t* corner_vertex_dev, float* grad_heights_dev,
                                           float* grad_cauchy_dev, void* scratch_dev, size_t scratch_bytes,
                                           pz_stream_t stream)
{
    if (!desc || desc->n_bins < 1 || !desc->etas)
        return fail(PZ_ERR_INVALID_ARGUMENT, "pz_adjoint_backward_compact: binned mode (etas, n_bins >= 1) required");
    if (!dloss_dspectral_dev || !corner_vertex_dev || !grad_heights_dev || !grad_cauchy_dev || !scratch_dev)
        return fail(PZ_ERR_INVALID_ARGUMENT, "pz_adjoint_backward_compact: null buffer");
    if (desc->cauchy_b == 0.0f)
        return fail(PZ_ERR_INVALID_ARGUMENT, "pz_adjoint_backward_compact: cauchy_b must be non-zero");
    if (scratch_bytes < pz_adjoint_scratch_bytes(1) || (reinterpret_cast<uintptr_t>(scratch_dev) & 255))
        return fail(PZ_ERR_SCRATCH_TOO_SMALL, "pz_adjoint_backward_compact: scratch too small or not 256-byte aligned");
    adjoint::AdjArgs a;
    int r = solve_args_from_desc(desc, &a.s, "pz_adjoint_backward_compact");
    if (r != PZ_OK) return r;
    a.s.nBins = desc->n_bins;
    a.s.etas = desc->etas;
    a.dLdI = dloss_dspectral_dev;
    a.corner = corner_vertex_dev;
    a.gradHeights = grad_heights_dev;
    a.gradCauchy = grad_cauchy_dev;
    char* base = static_cast<char*>(scratch_dev);
    auto* status = reinterpret_cast<uint32_t*>(base);
    auto* count = reinterpret_cast<unsigned long long*>(base + 8);
    auto* list = reinterpret_cast<adjoint::AdjRecord*>(base + kAdjHeader);
    const uint64_t capacity = (scratch_bytes - kAdjHeader) / sizeof(adjoint::AdjRecord);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(base, 0, 16, s);
    if (e == cudaSuccess) {
        switch (desc->K) {
            case 1: e = launch_adjoint_compact<1>(a, list, count, capacity, status, s); break;
            case 2: e = launch_adjoint_compact<2>(a, list, count, capacity, status, s); break;
            default:
                return fail(PZ_ERR_UNSUPPORTED, "pz_adjoint_backward_compact: K = %d (1 or 2 supported)", desc->K);
        }
    }
    if (e != cudaSuccess) return cuda_fail(e, "pz_adjoint_backward_compact");
    clear_error();
    return PZ_OK;
}
