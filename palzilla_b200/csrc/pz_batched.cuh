// pz_batched.cuh -- building blocks of the batched persistent specular solver.
//
// Multi-tangent forward-mode duals: one pass yields the constraint values and all 2K
// Jacobian columns (plus, optionally, the derivative with respect to eta), where the
// reference solver runs 2K single-tangent passes (pk.h:484-548).  Each tangent column
// is computed with exactly the operation sequence of a single-tangent pass, so the
// Jacobian equals the reference's column by column.
#pragma once
#include "pz_solver.cuh"

namespace pz {
namespace batched {

using namespace solver;
using pz::operator+;
using pz::operator-;
using pz::operator*;
using pz::operator/;

template <class T, int N> struct MD {
    T v;
    T g[N];
};
template <class T, int N> PZ_D MD<T, N> mconst(T v)
{
    MD<T, N> r;
    r.v = v;
#pragma unroll
    for (int i = 0; i < N; i++) r.g[i] = T(0);
    return r;
}
template <class T, int N> PZ_D MD<T, N> operator+(const MD<T, N>& a, const MD<T, N>& b)
{
    MD<T, N> r;
    r.v = a.v + b.v;
#pragma unroll
    for (int i = 0; i < N; i++) r.g[i] = a.g[i] + b.g[i];
    return r;
}
template <class T, int N> PZ_D MD<T, N> operator-(const MD<T, N>& a, const MD<T, N>& b)
{
    MD<T, N> r;
    r.v = a.v - b.v;
#pragma unroll
    for (int i = 0; i < N; i++) r.g[i] = a.g[i] - b.g[i];
    return r;
}
template <class T, int N> PZ_D MD<T, N> operator-(const MD<T, N>& a)
{
    MD<T, N> r;
    r.v = -a.v;
#pragma unroll
    for (int i = 0; i < N; i++) r.g[i] = -a.g[i];
    return r;
}
template <class T, int N> PZ_D MD<T, N> operator*(const MD<T, N>& a, const MD<T, N>& b)
{
    MD<T, N> r;
    r.v = a.v * b.v;
#pragma unroll
    for (int i = 0; i < N; i++) r.g[i] = a.g[i] * b.v + b.g[i] * a.v;
    return r;
}
template <class T, int N> PZ_D MD<T, N> operator/(const MD<T, N>& a, const MD<T, N>& b)
{
    MD<T, N> r;
    r.v = a.v / b.v;
    const T ib = T(1) / b.v, q = -a.v / (b.v * b.v);
#pragma unroll
    for (int i = 0; i < N; i++) r.g[i] = a.g[i] * ib + b.g[i] * q;
    return r;
}
template <class T, int N> PZ_D MD<T, N> msqrt(const MD<T, N>& a)
{
    MD<T, N> r;
    r.v = vsqrt(a.v);
    const T d = T(0.5) / vsqrt(a.v);
#pragma unroll
    for (int i = 0; i < N; i++) r.g[i] = a.g[i] * d;
    return r;
}
template <class T, int N> struct MD3 { MD<T, N> x, y, z; };
template <class T, int N> PZ_D MD3<T, N> m3(V3<T> v) { return {mconst<T, N>(v.x), mconst<T, N>(v.y), mconst<T, N>(v.z)}; }
template <class T, int N> PZ_D MD3<T, N> operator+(const MD3<T, N>& a, const MD3<T, N>& b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T, int N> PZ_D MD3<T, N> operator-(const MD3<T, N>& a, const MD3<T, N>& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T, int N> PZ_D MD3<T, N> operator-(const MD3<T, N>& a) { return {-a.x, -a.y, -a.z}; }
template <class T, int N> PZ_D MD3<T, N> operator*(const MD3<T, N>& a, const MD<T, N>& s) { return {a.x * s, a.y * s, a.z * s}; }
template <class T, int N> PZ_D MD3<T, N> operator/(const MD3<T, N>& a, const MD<T, N>& s) { return {a.x / s, a.y / s, a.z / s}; }
template <class T, int N> PZ_D MD<T, N> mdot(const MD3<T, N>& a, const MD3<T, N>& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T, int N> PZ_D MD3<T, N> mcross(const MD3<T, N>& a, const MD3<T, N>& b)
{
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// Constraint values c[3K] and Jacobian columns J[2K][3K] at params x (and, when
// kEta, dc/deta in J[2K]).  Same constraint as solve_constraints (pk.h:511-547).
template <class T, int K, bool kEta>
PZ_D void eval_constraints(const T* x, V3<T> p_beg, V3<T> p_end, const Chain<K>& ch, T eta, uint32_t events,
                           T (&J)[2 * K + (kEta ? 1 : 0)][3 * K], T (&c)[3 * K], T& cost)
{
    constexpr int N = 2 * K + (kEta ? 1 : 0);
    MD3<T, N> vtx[K + 2], sn[K];
    vtx[0] = m3<T, N>(p_beg);
    vtx[K + 1] = m3<T, N>(p_end);
#pragma unroll
    for (int k = 0; k < K; k++) {
        MD<T, N> pu = mconst<T, N>(x[2 * k]), pv = mconst<T, N>(x[2 * k + 1]);
        pu.g[2 * k] = T(1);
        pv.g[2 * k + 1] = T(1);
        vtx[k + 1] = m3<T, N>(v3f<T>(ch.v0[k])) + m3<T, N>(v3f<T>(ch.e0[k])) * pu + m3<T, N>(v3f<T>(ch.e1[k])) * pv;
        sn[k] = m3<T, N>(v3f<T>(ch.n0[k])) + m3<T, N>(v3f<T>(ch.ne0[k])) * pu + m3<T, N>(v3f<T>(ch.ne1[k])) * pv;
    }
    MD<T, N> em1 = mconst<T, N>(eta * eta - T(1));
    if (kEta) em1.g[N - 1] = T(2) * eta;
    cost = T(0);
#pragma unroll
    for (int k = 0; k < K; k++) {
        MD3<T, N> wi = vtx[k] - vtx[k + 1];
        MD3<T, N> wo = vtx[k + 2] - vtx[k + 1];
        const MD3<T, N> n = sn[k];
        if (mdot(wi, n).v < T(0)) {
            const MD3<T, N> t = wi;
            wi = wo;
            wo = t;
        }
        MD3<T, N> wopt;
        if ((events >> k) & 1u) {  // refraction_norm_free, saka.h:191-202
            const MD<T, N> NoN = mdot(n, n), WIoN = mdot(wi, n), WoW = mdot(wi, wi);
            const MD<T, N> kk = NoN * WoW * em1 + WIoN * WIoN;
            if (kk.v < T(0)) wopt = m3<T, N>(v3<T>(0, 0, 0));
            else wopt = -wi * NoN + n * (WIoN - msqrt(kk));
        } else {  // reflection, saka.h:186-189
            wopt = n * mdot(wi, n) * mconst<T, N>(T(2)) / mdot(n, n) - wi;
        }
        const MD3<T, N> cc = mcross(wo, wopt);
        c[3 * k + 0] = cc.x.v;
        c[3 * k + 1] = cc.y.v;
        c[3 * k + 2] = cc.z.v;
#pragma unroll
        for (int i = 0; i < N; i++) {
            J[i][3 * k + 0] = cc.x.g[i];
            J[i][3 * k + 1] = cc.y.g[i];
            J[i][3 * k + 2] = cc.z.g[i];
        }
        cost += cc.x.v * cc.x.v + cc.y.v * cc.y.v + cc.z.v * cc.z.v;
    }
}

// Householder QR least squares (same construction as solver::qr_solve) that also
// returns |det R| = prod |R_ii| (= sqrt(det(J^T J))).
template <class T, int R, int C>
PZ_D T qr_solve_det(T (&A)[C][R], T (&b)[R], T (&x)[C])
{
    constexpr int NH = (C < R - 1) ? C : R - 1;
    T vs[NH][R];
#pragma unroll
    for (int i = 0; i < NH; i++) {
        T cd = T(0);
#pragma unroll
        for (int j = 0; j < R; j++) {
            vs[i][j] = j < i ? T(0) : -A[i][j];
            cd += vs[i][j] * vs[i][j];
        }
        const T sgn = T(0) < vs[i][i] ? T(1) : T(-1);
        const T x_len = vsqrt(cd);
        vs[i][i] += sgn * x_len;
        const T v_len2 = T(2) * x_len * (x_len + fabs(A[i][i]));
        A[i][i] = sgn * x_len;
#pragma unroll
        for (int r = i + 1; r < R; r++) A[i][r] = T(0);
#pragma unroll
        for (int c = i + 1; c < C; c++) {
            T vdc = T(0);
#pragma unroll
            for (int r = i; r < R; r++) vdc += vs[i][r] * A[c][r];
            const T k = T(2) * vdc / v_len2;
#pragma unroll
            for (int r = i; r < R; r++) A[c][r] -= k * vs[i][r];
        }
    }
#pragma unroll
    for (int i = 0; i < NH; i++) {
        T vdc = T(0), vdv = T(0);
#pragma unroll
        for (int r = i; r < R; r++) {
            vdc += vs[i][r] * b[r];
            vdv += vs[i][r] * vs[i][r];
        }
        const T k = T(2) * vdc / vdv;
#pragma unroll
        for (int r = i; r < R; r++) b[r] -= k * vs[i][r];
    }
    T det = T(1);
#pragma unroll
    for (int r = C - 1; 0 <= r; r--) {
        T sum = T(0);
#pragma unroll
        for (int i = r + 1; i < C; i++) sum += A[i][r] * x[i];
        x[r] = (b[r] - sum) / A[r][r];
        det *= fabs(A[r][r]);
    }
    return det;
}

// Newton with the reference's rules (cost tolerance, edge rejection after the warm-up
// iterations) on the multi-tangent Jacobian.  Returns converged; *det = |det R| of
// the last factorisation (0 if none).
// relative determinant of R: prod_i |R_ii| / max_i |R_ii|^C (scale-free; 1 = well conditioned)
template <class T, int R, int C>
PZ_D T qr_solve_reldet(T (&A)[C][R], T (&b)[R], T (&x)[C])
{
    T scale = T(0);
    const T det = qr_solve_det<T, R, C>(A, b, x);
#pragma unroll
    for (int i = 0; i < C; i++) scale = fmax(scale, fabs(A[i][i]));
    T s = T(1);
#pragma unroll
    for (int i = 0; i < C; i++) s *= scale;
    return s > T(0) ? det / s : T(0);
}

// minSteps: Newton steps taken before the cost test may stop the iteration (a warm start
// inside the tolerance still gets quadratically refined).
template <class T, int K>
PZ_D bool newton(T* x, V3<T> p_beg, V3<T> p_end, const Chain<K>& ch, T eta, uint32_t events, int maxIter, T tol,
                 int warmup, bool edgeRejection, int* iters, T* det, int minSteps = 0)
{
    T edge_eps = T(0.25);
    *det = T(1);  // no factorisation taken: treated as well conditioned
    for (int iter = 0; iter < maxIter; iter++) {
        T J[2 * K][3 * K], c[3 * K], cost;
        eval_constraints<T, K, false>(x, p_beg, p_end, ch, eta, events, J, c, cost);
        if (cost < tol && iter >= minSteps) {
            *iters = iter;
            return true;
        }
        T dx[2 * K];
        *det = qr_solve_reldet<T, 3 * K, 2 * K>(J, c, dx);
#pragma unroll
        for (int i = 0; i < 2 * K; i++) x[i] = x[i] - dx[i];
        if (edgeRejection && warmup <= iter) {
#pragma unroll
            for (int k = 0; k < K; k++) {
                const T u = x[2 * k], v = x[2 * k + 1];
                if (!(-edge_eps < u && -edge_eps < v && u + v < T(1) + edge_eps)) {
                    *iters = iter + 1;
                    return false;
                }
            }
            edge_eps *= edge_eps;
        }
        // diverged: not finite
        if (!(fabs(x[0]) < T(1.0e6))) {
            *iters = iter + 1;
            return false;
        }
    }
    *iters = maxIter;
    return false;
}


// dAdw (pk.h:844-930) with both ray-differential tangents carried in one pass; each
// tangent follows the single-tangent operation sequence of the reference.
template <class T, int K>
PZ_D T dadw2(V3<T> ro, V3<T> rd, V3<T> p_end, const Chain<K>& ch, uint32_t events, T eta)
{
    rd = vnormalize(rd);
    const T sign = copysign(T(1), rd.z);
    const T a = T(-1) / (sign + rd.z);
    const T bb = rd.x * rd.y * a;
    const V3<T> T0 = v3<T>(T(1) + sign * rd.x * rd.x * a, sign * bb, -sign * rd.x);
    const V3<T> T1 = v3<T>(bb, sign + rd.y * rd.y * a, -rd.y);
    MD<T, 2> d0 = mconst<T, 2>(T(0)), d1 = mconst<T, 2>(T(0));
    d0.g[0] = T(1);
    d1.g[1] = T(1);
    MD3<T, 2> ro_j = m3<T, 2>(ro);
    MD3<T, 2> rd_j = m3<T, 2>(rd) + m3<T, 2>(T0) * d0 + m3<T, 2>(T1) * d1;
#pragma unroll
    for (int j = 0; j < K; j++) {
        const V3<T> ng = v3f<T>(ch.ng[j]);
        const V3<T> tv0 = v3f<T>(ch.v0[j]);
        const V3<T> tv1 = tv0 + v3f<T>(ch.e0[j]);
        const V3<T> tv2 = tv0 + v3f<T>(ch.e1[j]);
        const MD<T, 2> t = mdot(m3<T, 2>(tv0) - ro_j, m3<T, 2>(ng)) / mdot(m3<T, 2>(ng), rd_j);
        const MD3<T, 2> p = ro_j + rd_j * t;
        MD<T, 2> v = mdot(p - m3<T, 2>(tv1), m3<T, 2>(vcross(ng, tv1 - tv0)));
        MD<T, 2> w = mdot(p - m3<T, 2>(tv2), m3<T, 2>(vcross(ng, tv2 - tv1)));
        MD<T, 2> u = mdot(p - m3<T, 2>(tv0), m3<T, 2>(vcross(ng, tv0 - tv2)));
        const MD<T, 2> area = u + v + w;
        u = u / area;
        v = v / area;
        w = w / area;
        const V3<T> n0 = v3f<T>(ch.n0[j]);
        const V3<T> n1 = n0 + v3f<T>(ch.ne0[j]);
        const V3<T> n2 = n0 + v3f<T>(ch.ne1[j]);
        const MD3<T, 2> n = m3<T, 2>(n0) * w + m3<T, 2>(n1) * u + m3<T, 2>(n2) * v;
        const MD3<T, 2> wi = -rd_j;
        MD3<T, 2> wo;
        auto refr = [](const MD3<T, 2>& wv, const MD3<T, 2>& nv, T e, bool& tir) {
            const MD<T, 2> NoN = mdot(nv, nv), WIoN = mdot(wv, nv), WoW = mdot(wv, wv);
            const MD<T, 2> kk = NoN * WoW * mconst<T, 2>(e * e - T(1)) + WIoN * WIoN;
            tir = kk.v < T(0);
            if (tir) return m3<T, 2>(v3<T>(0, 0, 0));
            return -wv * NoN + nv * (WIoN - msqrt(kk));
        };
        if ((events >> j) & 1u) {
            bool tir;
            if (mdot(wi, n).v < T(0)) {
                wo = refr(wi, -n, T(1) / eta, tir);
                if (tir) return T(3.402823466e+38f);
            } else {
                wo = refr(wi, n, eta, tir);
            }
        } else {
            wo = n * mdot(wi, n) * mconst<T, 2>(T(2)) / mdot(n, n) - wi;
        }
        ro_j = p;
        rd_j = wo;
    }
    const V3<T> p_last = v3<T>(ro_j.x.v, ro_j.y.v, ro_j.z.v);
    const MD3<T, 2> pn = m3<T, 2>(p_last - p_end);
    const MD<T, 2> t = mdot(m3<T, 2>(p_end) - ro_j, pn) / mdot(pn, rd_j);
    const MD3<T, 2> pf = ro_j + rd_j * t;
    const V3<T> ax0 = v3<T>(pf.x.g[0], pf.y.g[0], pf.z.g[0]), ax1 = v3<T>(pf.x.g[1], pf.y.g[1], pf.z.g[1]);
    const T len0 = vlength(ax0), len1 = vlength(ax1);
    const T s = vlength(vcross(ax0 / len0, ax1 / len1));
    return len0 * len1 * vfmax(s, T(0.01));
}

// position of the k-th (0-based) set bit of a 64-bit mask
PZ_D int nth_bit64(unsigned long long m, int k)
{
    const uint32_t lo = (uint32_t)m;
    const int c = __popc(lo);
    if (k < c) return (int)__fns(lo, 0, k + 1);
    return 32 + (int)__fns((uint32_t)(m >> 32), 0, k - c + 1);
}

}  // namespace batched
}  // namespace pz
