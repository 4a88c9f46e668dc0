// pz_solver.cuh -- specular-constraint solver on the device.
//
// solve_constraints<T, K>: Gauss-Newton on the 3K normalisation-free constraints
// c_k = cross(wo_k, refract/reflect(wi_k, n_k)) over the 2K barycentrics of a
// K-vertex specular chain, with the Jacobian from 2K forward-mode passes and the step
// from a Householder-QR least-squares solve; early rejection when a vertex leaves its
// triangle by more than edge_eps (0.25, squared after every warm-up iteration).  This is
// solveConstraints<K> (pk.h:466-592) with saka's dual numbers (saka.h:11-202) and
// sen's solve_qr_overdetermined (sen.h:658-747), restated for T = float (the product
// solver) and T = double (the FP64 polish).
// contributable_throughput<T, K>: contributableThroughput<K> (pk.h:760-842).
// dadw<T>: dAdw (pk.h:844-930).
#pragma once
#include "pz_optics.cuh"
#include "pz_trace.cuh"

namespace pz {
namespace solver {

// float3 operators of namespace pz (hidden by the V3 / dual templates below otherwise)
using pz::operator+;
using pz::operator-;
using pz::operator*;
using pz::operator/;

template <class T> struct V3 { T x, y, z; };
template <class T> PZ_HD V3<T> v3(T x, T y, T z) { return V3<T>{x, y, z}; }
template <class T> PZ_HD V3<T> v3f(float3 a) { return V3<T>{(T)a.x, (T)a.y, (T)a.z}; }
template <class T> PZ_HD V3<T> operator+(V3<T> a, V3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T> PZ_HD V3<T> operator-(V3<T> a, V3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T> PZ_HD V3<T> operator-(V3<T> a) { return {-a.x, -a.y, -a.z}; }
template <class T> PZ_HD V3<T> operator*(V3<T> a, T s) { return {a.x * s, a.y * s, a.z * s}; }
template <class T> PZ_HD V3<T> operator/(V3<T> a, T s) { return {a.x / s, a.y / s, a.z / s}; }
template <class T> PZ_HD T vdot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> PZ_HD V3<T> vcross(V3<T> a, V3<T> b)
{
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class T> PZ_D T vsqrt(T x) { return sqrt(x); }
template <> PZ_D float vsqrt<float>(float x) { return sqrtf(x); }
template <class T> PZ_D T vlength(V3<T> a) { return vsqrt(vdot(a, a)); }
template <class T> PZ_D V3<T> vnormalize(V3<T> a) { return a * (T(1) / vsqrt(vdot(a, a))); }
template <class T> PZ_D T vfmax(T a, T b) { return a > b ? a : (b != b ? a : b); }

// ---------------------------------------------------------------- forward-mode duals
template <class T> struct D { T v, g; };
template <class T> PZ_HD D<T> dc(T v) { return D<T>{v, T(0)}; }
template <class T> PZ_HD D<T> operator+(D<T> a, D<T> b) { return {a.v + b.v, a.g + b.g}; }
template <class T> PZ_HD D<T> operator-(D<T> a, D<T> b) { return {a.v - b.v, a.g - b.g}; }
template <class T> PZ_HD D<T> operator-(D<T> a) { return {-a.v, -a.g}; }
template <class T> PZ_HD D<T> operator*(D<T> a, D<T> b) { return {a.v * b.v, a.g * b.v + b.g * a.v}; }
template <class T> PZ_HD D<T> operator/(D<T> a, D<T> b)  // saka.h:77-83
{
    return {a.v / b.v, a.g * (T(1) / b.v) + b.g * (-a.v / (b.v * b.v))};
}
template <class T> PZ_D D<T> dsqrt(D<T> a)
{
    const T s = vsqrt(a.v);
    return {s, a.g * (T(0.5) / s)};
}
template <class T> struct D3 { D<T> x, y, z; };
template <class T> PZ_HD D3<T> d3(V3<T> v) { return {dc(v.x), dc(v.y), dc(v.z)}; }
template <class T> PZ_HD D3<T> operator+(D3<T> a, D3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T> PZ_HD D3<T> operator-(D3<T> a, D3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T> PZ_HD D3<T> operator-(D3<T> a) { return {-a.x, -a.y, -a.z}; }
template <class T> PZ_HD D3<T> operator*(D3<T> a, D<T> s) { return {a.x * s, a.y * s, a.z * s}; }
template <class T> PZ_HD D3<T> operator/(D3<T> a, D<T> s) { return {a.x / s, a.y / s, a.z / s}; }
template <class T> PZ_HD D<T> ddot(D3<T> a, D3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> PZ_HD D3<T> dcross(D3<T> a, D3<T> b)
{
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class T> PZ_HD D3<T> dreflection(D3<T> wi, D3<T> n) { return n * ddot(wi, n) * dc(T(2)) / ddot(n, n) - wi; }
template <class T> PZ_D D3<T> drefraction(D3<T> wi, D3<T> n, T eta)
{
    const D<T> NoN = ddot(n, n), WIoN = ddot(wi, n), WoW = ddot(wi, wi);
    const D<T> k = NoN * WoW * dc(eta * eta - T(1)) + WIoN * WIoN;
    if (k.v < T(0)) return d3(v3<T>(0, 0, 0));
    return -wi * NoN + n * (WIoN - dsqrt(k));
}

// ---------------------------------------------------------------- scene records of a tuple
template <int K> struct Chain {
    float3 v0[K], e0[K], e1[K];   // triangle vertex 0 and edges
    float3 n0[K], ne0[K], ne1[K]; // shading normal at vertex 0 and its edges
    float3 ng[K];                 // unnormalised geometric normal
    int32_t material[K];
};

template <int K>
PZ_D void load_chain(Chain<K>& c, const Tri* __restrict__ tris, const Attrib* __restrict__ attribs, const int* idx)
{
#pragma unroll
    for (int k = 0; k < K; k++) {
        float3 a, b, d;
        load_tri(tris, (uint32_t)idx[k], a, b, d);
        c.v0[k] = a;
        c.e0[k] = b - a;
        c.e1[k] = d - a;
        c.ng[k] = cross(b - a, d - a);
        const float* sn = reinterpret_cast<const float*>(attribs + idx[k]) + 1;
        const float3 n0 = mk3(__ldg(sn + 0), __ldg(sn + 1), __ldg(sn + 2));
        const float3 n1 = mk3(__ldg(sn + 3), __ldg(sn + 4), __ldg(sn + 5));
        const float3 n2 = mk3(__ldg(sn + 6), __ldg(sn + 7), __ldg(sn + 8));
        c.n0[k] = n0;
        c.ne0[k] = n1 - n0;
        c.ne1[k] = n2 - n0;
        c.material[k] = __ldg(&attribs[idx[k]].material);
    }
}

// The chain of triangles and attributes given by value (the reference's solver arguments).
template <int K>
PZ_D void make_chain(Chain<K>& c, const Tri* tris, const Attrib* attribs)
{
#pragma unroll
    for (int k = 0; k < K; k++) {
        const float3 a = tris[k].v0, b = tris[k].v1, d = tris[k].v2;
        c.v0[k] = a;
        c.e0[k] = b - a;
        c.e1[k] = d - a;
        c.ng[k] = cross(b - a, d - a);
        c.n0[k] = attribs[k].n0;
        c.ne0[k] = attribs[k].n1 - attribs[k].n0;
        c.ne1[k] = attribs[k].n2 - attribs[k].n0;
        c.material[k] = attribs[k].material;
    }
}

// ---------------------------------------------------------------- Householder QR least squares
// Solves min |A x - b| for A (R x C, column-major, R >= C) by the reference's
// Householder construction (sen.h:658-747).
template <class T, int R, int C>
PZ_D void qr_solve(T (&A)[C][R], T (&b)[R], T (&x)[C])
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
#pragma unroll
    for (int r = C - 1; 0 <= r; r--) {
        T sum = T(0);
#pragma unroll
        for (int i = r + 1; i < C; i++) sum += A[i][r] * x[i];
        x[r] = (b[r] - sum) / A[r][r];
    }
}

// ---------------------------------------------------------------- Newton solve
// The end-of-iteration callback of solveConstraints (pk.h:461-463): called with
// (iteration, true) when the cost test passes, and with (iteration, iteration ==
// maxIterations - 1) after every other iteration that is not rejected at a triangle edge.
struct NoCallback {
    PZ_D void operator()(int, bool) const {}
};

template <class T, int K, class Callback = NoCallback>
PZ_D bool solve_constraints(T* params, V3<T> p_beg, V3<T> p_end, const Chain<K>& ch, T eta, uint32_t events,
                            int maxIterations, T costTolerance, int earlyTermWarmUp, int* itersOut = nullptr,
                            Callback end_of_iter = Callback())
{
    constexpr int NP = 2 * K;
    T edge_eps = T(0.25);
    for (int iter = 0; iter < maxIterations; iter++) {
        T A[NP][3 * K];
        T b[3 * K];
        T cost = T(0);
#pragma unroll
        for (int i = 0; i < NP; i++) {
            D3<T> vtx[K + 2];
            D3<T> sn[K];
            vtx[0] = d3(p_beg);
            vtx[K + 1] = d3(p_end);
#pragma unroll
            for (int k = 0; k < K; k++) {
                const D<T> pu{params[2 * k + 0], T(2 * k + 0 == i ? 1 : 0)};
                const D<T> pv{params[2 * k + 1], T(2 * k + 1 == i ? 1 : 0)};
                vtx[k + 1] = d3(v3f<T>(ch.v0[k])) + d3(v3f<T>(ch.e0[k])) * pu + d3(v3f<T>(ch.e1[k])) * pv;
                sn[k] = d3(v3f<T>(ch.n0[k])) + d3(v3f<T>(ch.ne0[k])) * pu + d3(v3f<T>(ch.ne1[k])) * pv;
            }
#pragma unroll
            for (int k = 0; k < K; k++) {
                D3<T> wi = vtx[k] - vtx[k + 1];
                D3<T> wo = vtx[k + 2] - vtx[k + 1];
                const D3<T> n = sn[k];
                if (ddot(wi, n).v < T(0)) {
                    const D3<T> t = wi;
                    wi = wo;
                    wo = t;
                }
                const D3<T> wopt = ((events >> k) & 1u) ? drefraction(wi, n, eta) : dreflection(wi, n);
                const D3<T> c = dcross(wo, wopt);
                A[i][3 * k + 0] = c.x.g;
                A[i][3 * k + 1] = c.y.g;
                A[i][3 * k + 2] = c.z.g;
                b[3 * k + 0] = c.x.v;
                b[3 * k + 1] = c.y.v;
                b[3 * k + 2] = c.z.v;
                if (i == 0) cost += c.x.v * c.x.v + c.y.v * c.y.v + c.z.v * c.z.v;
            }
        }
        if (cost < costTolerance) {
            if (itersOut) *itersOut = iter;
            end_of_iter(iter, true);
            return true;
        }
        T dp[NP];
        qr_solve<T, 3 * K, NP>(A, b, dp);
#pragma unroll
        for (int i = 0; i < NP; i++) params[i] = params[i] - dp[i];
        if (earlyTermWarmUp <= iter) {
#pragma unroll
            for (int k = 0; k < K; k++) {
                const T u = params[2 * k], v = params[2 * k + 1];
                if (!(-edge_eps < u && -edge_eps < v && u + v < T(1) + edge_eps)) {
                    if (itersOut) *itersOut = iter + 1;
                    return false;
                }
            }
            edge_eps *= edge_eps;
        }
        end_of_iter(iter, iter == maxIterations - 1);
    }
    if (itersOut) *itersOut = maxIterations;
    return false;
}

template <class T, int K> PZ_D V3<T> vertex(const Chain<K>& ch, const T* params, int k)
{
    return v3f<T>(ch.v0[k]) + v3f<T>(ch.e0[k]) * params[2 * k] + v3f<T>(ch.e1[k]) * params[2 * k + 1];
}

template <class T>
PZ_D T fresnel_T(V3<T> wi, V3<T> n, T eta)
{
    T nn = vdot(n, n), wiwi = vdot(wi, wi), C = vdot(n, wi);
    if (C < T(0)) {
        C = -C;
        n = -n;
        eta = T(1) / eta;
    }
    const T K2 = nn * wiwi * (eta * eta - T(1)) + C * C;
    if (K2 < T(0)) return T(1);
    const T G = vsqrt(K2);
    const T GmC = G - C, GpC = G + C;
    const T a = GmC / GpC, b = (C * GpC - nn * wiwi) / (C * GmC + nn * wiwi);
    return T(0.5) * (a * a) * (T(1) + b * b);
}

// contributableThroughput<K>, pk.h:760-842 (visibility through the float BVH)
template <class T, int K>
PZ_D T contributable_throughput(const T* params, V3<T> p_beg, V3<T> p_end, const Chain<K>& ch, uint32_t events,
                                const Node* nodes, const Tri* tris, uint32_t root, T eta)
{
    V3<T> vtx[K + 2], sn[K + 2];
    vtx[0] = p_beg;
    vtx[K + 1] = p_end;
#pragma unroll
    for (int k = 0; k < K; k++) {
        const T u = params[2 * k], v = params[2 * k + 1];
        if (u < T(0) || v < T(0) || T(1) < u + v) return T(0);
        vtx[k + 1] = vertex<T, K>(ch, params, k);
        sn[k + 1] = vnormalize(v3f<T>(ch.n0[k]) + v3f<T>(ch.ne0[k]) * u + v3f<T>(ch.ne1[k]) * v);
    }
    sn[0] = vnormalize(vtx[1] - vtx[0]);
    sn[K + 1] = vnormalize(vtx[K] - vtx[K + 1]);
    T thr = T(1);
#pragma unroll
    for (int k = 0; k < K; k++) {
        const V3<T> wi = vtx[k] - vtx[k + 1], wo = vtx[k + 2] - vtx[k + 1], n = sn[k + 1];
        const bool eR = T(0) < vdot(wi, n) * vdot(wo, n);
        if (((events >> k) & 1u) == (eR ? 1u : 0u)) return T(0);
        const V3<T> ng = v3f<T>(ch.ng[k]);
        const bool egR = T(0) < vdot(wi, ng) * vdot(wo, ng);
        if (eR != egR) return T(0);
        if (ch.material[k] == kDielectric) {
            const T r = fresnel_T(wi, n, eta);
            thr *= eR ? r : T(1) - r;
        }
    }
#pragma unroll
    for (int i = 0; i < K + 1; i++) {
        const V3<T> dd = vtx[i] - vtx[i + 1];
        if (vdot(dd, dd) < T(1.0e-5f)) return T(0);
    }
#pragma unroll 1
    for (int i = 0; i < K + 1; i++) {
        const float3 a = mk3((float)vtx[i].x, (float)vtx[i].y, (float)vtx[i].z);
        const float3 b = mk3((float)vtx[i + 1].x, (float)vtx[i + 1].y, (float)vtx[i + 1].z);
        const float3 na = mk3((float)sn[i].x, (float)sn[i].y, (float)sn[i].z);
        const float3 nb = mk3((float)sn[i + 1].x, (float)sn[i + 1].y, (float)sn[i + 1].z);
        if (occluded(nodes, tris, root, a, na, b, nb)) return T(0);
    }
    return thr;
}

// dAdw, pk.h:844-930: generalized geometry term by ray differentials through the chain
template <class T, int K>
PZ_D T dadw(V3<T> ro, V3<T> rd, V3<T> p_end, const Chain<K>& ch, uint32_t events, T eta)
{
    rd = vnormalize(rd);
    V3<T> dAxis[2];
#pragma unroll
    for (int i = 0; i < 2; i++) {
        D<T> dif[2] = {dc(T(0)), dc(T(0))};
        dif[i].g = T(1);
        D3<T> ro_j = d3(ro);
        const T sign = copysign(T(1), rd.z);  // GetOrthonormalBasis, pk.h:453-459
        const T a = T(-1) / (sign + rd.z);
        const T bb = rd.x * rd.y * a;
        const V3<T> T0 = v3<T>(T(1) + sign * rd.x * rd.x * a, sign * bb, -sign * rd.x);
        const V3<T> T1 = v3<T>(bb, sign + rd.y * rd.y * a, -rd.y);
        D3<T> rd_j = d3(rd) + d3(T0) * dif[0] + d3(T1) * dif[1];
#pragma unroll
        for (int j = 0; j < K; j++) {
            const V3<T> ng = v3f<T>(ch.ng[j]);
            const V3<T> tv0 = v3f<T>(ch.v0[j]);
            const V3<T> tv1 = tv0 + v3f<T>(ch.e0[j]);
            const V3<T> tv2 = tv0 + v3f<T>(ch.e1[j]);
            const D<T> t = ddot(d3(tv0) - ro_j, d3(ng)) / ddot(d3(ng), rd_j);
            const D3<T> p = ro_j + rd_j * t;
            D<T> v = ddot(p - d3(tv1), d3(vcross(ng, tv1 - tv0)));
            D<T> w = ddot(p - d3(tv2), d3(vcross(ng, tv2 - tv1)));
            D<T> u = ddot(p - d3(tv0), d3(vcross(ng, tv0 - tv2)));
            const D<T> area = u + v + w;
            u = u / area;
            v = v / area;
            w = w / area;
            const V3<T> n0 = v3f<T>(ch.n0[j]);
            const V3<T> n1 = n0 + v3f<T>(ch.ne0[j]);
            const V3<T> n2 = n0 + v3f<T>(ch.ne1[j]);
            const D3<T> n = d3(n0) * w + d3(n1) * u + d3(n2) * v;
            const D3<T> wi = -rd_j;
            D3<T> wo;
            if ((events >> j) & 1u) {
                if (ddot(wi, n).v < T(0)) {
                    wo = drefraction(wi, -n, T(1) / eta);
                    if (wo.x.v == T(0) && wo.y.v == T(0) && wo.z.v == T(0)) return T(3.402823466e+38f);
                } else {
                    wo = drefraction(wi, n, eta);
                }
            } else {
                wo = dreflection(wi, n);
            }
            ro_j = p;
            rd_j = wo;
        }
        const V3<T> p_last = v3<T>(ro_j.x.v, ro_j.y.v, ro_j.z.v);
        const D3<T> pn = d3(p_last - p_end);
        const D<T> t = ddot(d3(p_end) - ro_j, pn) / ddot(pn, rd_j);
        const D3<T> pf = ro_j + rd_j * t;
        dAxis[i] = v3<T>(pf.x.g, pf.y.g, pf.z.g);
    }
    const T len0 = vlength(dAxis[0]), len1 = vlength(dAxis[1]);
    const T s = vlength(vcross(dAxis[0] / len0, dAxis[1] / len1));
    return len0 * len1 * vfmax(s, T(0.01));
}

}  // namespace solver
}  // namespace pz
