// pz_oracle_flops.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Counts the floating-point operations of one Newton iteration of the restated
// solveConstraints<K> (pk.h:466-592; pz_oracle.hpp solve_constraints) by running it with a
// counting scalar type: every +, -, *, / and sqrt on the scalar adds one to its counter
// (negation, fabs and comparisons are not counted).  One iteration is the 2K dual
// evaluations of the constraints (one per barycentric: the reference's single-tangent
// Jacobian columns), the Householder QR least-squares step and the update.  Used by
// bench.py's CPU-baseline leg to state the solve's FP32 operations per second.
#include <cmath>
#include <cstdint>

namespace pzo_flops {
struct Counts {
    unsigned long long add, mul, div, sqrt;
};
static Counts g_counts;

// float with operation counts
struct CF {
    float v;
    CF() : v(0.0f) {}
    CF(float x) : v(x) {}
    CF(double x) : v((float)x) {}
    CF(int x) : v((float)x) {}
};
inline CF operator+(CF a, CF b) { g_counts.add++; return CF(a.v + b.v); }
inline CF operator-(CF a, CF b) { g_counts.add++; return CF(a.v - b.v); }
inline CF operator-(CF a) { return CF(-a.v); }
inline CF operator*(CF a, CF b) { g_counts.mul++; return CF(a.v * b.v); }
inline CF operator/(CF a, CF b) { g_counts.div++; return CF(a.v / b.v); }
inline CF& operator+=(CF& a, CF b) { a = a + b; return a; }
inline CF& operator-=(CF& a, CF b) { a = a - b; return a; }
inline CF& operator*=(CF& a, CF b) { a = a * b; return a; }
inline bool operator<(CF a, CF b) { return a.v < b.v; }
inline bool operator>(CF a, CF b) { return a.v > b.v; }
inline bool operator<=(CF a, CF b) { return a.v <= b.v; }
inline bool operator>=(CF a, CF b) { return a.v >= b.v; }
}  // namespace pzo_flops

// The restatement calls std::sqrt / std::fabs on its scalar type; these overloads are
// declared before its templates so that they are found when it is instantiated with CF.
namespace std {
inline pzo_flops::CF sqrt(pzo_flops::CF a) { pzo_flops::g_counts.sqrt++; return pzo_flops::CF(std::sqrt(a.v)); }
inline pzo_flops::CF fabs(pzo_flops::CF a) { return pzo_flops::CF(std::fabs(a.v)); }
inline pzo_flops::CF fmax(pzo_flops::CF a, pzo_flops::CF b) { return pzo_flops::CF(std::fmax(a.v, b.v)); }
inline pzo_flops::CF fmin(pzo_flops::CF a, pzo_flops::CF b) { return pzo_flops::CF(std::fmin(a.v, b.v)); }
}  // namespace std

#include "pz_oracle.hpp"

using pzo_flops::CF;

template <int K>
static void one_iteration(const float* params, const float* p_beg, const float* p_end, const pzo::Triangle* tris,
                          const pzo::TriangleAttrib* attribs, float eta, uint32_t events)
{
    CF x[2 * K];
    for (int i = 0; i < 2 * K; i++) x[i] = CF(params[i]);
    const pzo::V3<CF> a{CF(p_beg[0]), CF(p_beg[1]), CF(p_beg[2])};
    const pzo::V3<CF> b{CF(p_end[0]), CF(p_end[1]), CF(p_end[2])};
    // one iteration: the cost is never below a tolerance of 0, and the edge test starts
    // after the last iteration
    pzo::solve_constraints<CF, K>(x, a, b, tris, attribs, CF(eta), events, 1, CF(0.0f), 1 << 20);
}

// Operation counts of one Newton iteration of the K-vertex chain: out[0..4) = additions and
// subtractions, multiplications, divisions, square roots.  Returns 0, or -1 for a bad K.
extern "C" int pzo_count_newton_flops(int K, const float* params, const float* p_beg, const float* p_end,
                                      const void* tris, const void* attribs, float eta, uint32_t events,
                                      unsigned long long* out)
{
    pzo_flops::g_counts = pzo_flops::Counts{0, 0, 0, 0};
    const auto* t = static_cast<const pzo::Triangle*>(tris);
    const auto* at = static_cast<const pzo::TriangleAttrib*>(attribs);
    switch (K) {
        case 1: one_iteration<1>(params, p_beg, p_end, t, at, eta, events); break;
        case 2: one_iteration<2>(params, p_beg, p_end, t, at, eta, events); break;
        case 3: one_iteration<3>(params, p_beg, p_end, t, at, eta, events); break;
        case 4: one_iteration<4>(params, p_beg, p_end, t, at, eta, events); break;
        default: return -1;
    }
    out[0] = pzo_flops::g_counts.add;
    out[1] = pzo_flops::g_counts.mul;
    out[2] = pzo_flops::g_counts.div;
    out[3] = pzo_flops::g_counts.sqrt;
    return 0;
}
