// palzilla_b200_device.cuh -- device-callable specular-constraint solver with the
// reference's signature, for CUDA code that solves specular chains inside its own kernels.
//
// Replaces solveConstraints<K> (pk.h:466-592) and its types EventDescriptor (pk.h:122-162)
// and SolverEmptyCallback (pk.h:461-463):
//
//   template <int K, class callback = SolverEmptyCallback>
//   __device__ bool solveConstraints(float parameters[K * 2], float3 p_beg, float3 p_end,
//                                    pz_triangle tris[K], pz_triangle_attrib attribs[K], float eta,
//                                    EventDescriptor eDescriptor, int maxIterations,
//                                    float costTolerance, int earlyTermWarmUp,
//                                    callback end_of_iter = SolverEmptyCallback());
//
// Gauss-Newton on the 3K normalisation-free constraints cross(wo_k, refract/reflect(wi_k,
// n_k)) of the K-vertex chain from p_beg (the light) to p_end (the receiver point), over
// the 2K barycentrics in `parameters` (the start on entry, the last iterate on return),
// with the Jacobian by forward-mode duals and the step by Householder-QR least squares.
// Returns true when the cost fell below costTolerance; false when a vertex left its
// triangle by more than the shrinking edge margin after earlyTermWarmUp iterations, or
// after maxIterations.  end_of_iter(iter, converged) is called as the reference calls it:
// with (iter, true) on convergence and with (iter, iter == maxIterations - 1) after every
// other iteration that is not rejected at an edge.  pz_triangle and pz_triangle_attrib are
// the reference's Triangle (36 B) and TriangleAttrib (40 B); bit k of the event descriptor
// set means transmission (refraction) at vertex k, else reflection.
//
// Compile the translation unit with -fmad=false for results equal to the reference's CPU
// float arithmetic bit for bit; with contraction the roots agree to rounding, while accept /
// reject decisions of marginal paths can differ.  Include with -I<repository>/include; the
// solver templates come from palzilla_b200/csrc.  pz_solve_constraints (palzilla_b200.h)
// runs this function over a batch from the library.
#pragma once
#include <cuda_runtime.h>

#include "palzilla_b200.h"
#include "../palzilla_b200/csrc/pz_solver.cuh"

namespace palzilla_b200 {

// EventDescriptor, pk.h:122-162: 24 event bits (1 = T, 0 = R) and the chain length.
struct EventDescriptor {
    uint32_t m_events : 24;
    uint32_t m_size : 8;
    __host__ __device__ EventDescriptor() : m_events(0), m_size(0) {}
    __host__ __device__ static EventDescriptor fromU32(uint32_t u)
    {
        EventDescriptor e;
        e.m_events = u & 0xFFFFFFu;
        e.m_size = u >> 24;
        return e;
    }
    __host__ __device__ bool isTransmission(uint32_t index) const { return (m_events >> index) & 1u; }
    __host__ __device__ int size() const { return m_size; }
    __host__ __device__ uint32_t asU32() const { return ((uint32_t)m_size << 24) | m_events; }
};
static_assert(sizeof(EventDescriptor) == 4, "EventDescriptor is one 32-bit word");

struct SolverEmptyCallback {
    __device__ void operator()(int, bool) const {}
};

template <int K, class callback = SolverEmptyCallback>
__device__ inline bool solveConstraints(float parameters[K * 2], float3 p_beg, float3 p_end, pz_triangle tris[K],
                                        pz_triangle_attrib attribs[K], float eta, EventDescriptor eDescriptor,
                                        int maxIterations, float costTolerance, int earlyTermWarmUp,
                                        callback end_of_iter = SolverEmptyCallback())
{
    static_assert(K >= 1 && K <= 4, "chains of 1 to 4 specular vertices");
    static_assert(sizeof(pz_triangle) == sizeof(pz::Tri) && sizeof(pz_triangle_attrib) == sizeof(pz::Attrib),
                  "reference layouts");
    pz::solver::Chain<K> ch;
    pz::solver::make_chain<K>(ch, reinterpret_cast<const pz::Tri*>(tris), reinterpret_cast<const pz::Attrib*>(attribs));
    return pz::solver::solve_constraints<float, K>(parameters, pz::solver::v3f<float>(p_beg),
                                                   pz::solver::v3f<float>(p_end), ch, eta, eDescriptor.asU32(),
                                                   maxIterations, costTolerance, earlyTermWarmUp, nullptr, end_of_iter);
}

}  // namespace palzilla_b200
