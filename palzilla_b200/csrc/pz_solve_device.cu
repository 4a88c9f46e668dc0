// pz_solve_device.cu -- pz_solve_constraints: a batch of device-side solveConstraints<K>
// calls (pk.h:466-592) through the public device-callable solver
// (include/palzilla_b200_device.cuh), one thread per item.  Built without FMA contraction,
// so every root equals the reference's CPU float arithmetic bit for bit.
#include "../../include/palzilla_b200_device.cuh"
#include "pz_capi_internal.h"

namespace pz {
namespace {

int done(cudaError_t e, const char* where)
{
    if (e != cudaSuccess) return cuda_fail(e, where);
    clear_error();
    return PZ_OK;
}

// The last iteration reported to the end-of-iteration callback.
struct LastIteration {
    int* last;
    __device__ void operator()(int iter, bool) const { *last = iter; }
};

template <int K>
__global__ void __launch_bounds__(256) k_solve_constraints(uint32_t events, float3 p_beg,
                                                           const int32_t* __restrict__ tuples,
                                                           const float3* __restrict__ p_end,
                                                           const float* __restrict__ etas, uint32_t n,
                                                           const pz_triangle* __restrict__ tris,
                                                           const pz_triangle_attrib* __restrict__ attribs,
                                                           uint32_t nTris, int maxIterations, float costTolerance, int warmup,
                                                           float* __restrict__ params, uint8_t* __restrict__ converged,
                                                           int32_t* __restrict__ iters)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    pz_triangle tk[K];
    pz_triangle_attrib ak[K];
    bool valid = true;
#pragma unroll
    for (int k = 0; k < K; k++) valid = valid && (uint32_t)tuples[(size_t)i * K + k] < nTris;
    if (!valid) {  // a triangle index out of range: the item is not solved
        if (converged) converged[i] = 0;
        if (iters) iters[i] = -2;
        return;
    }
#pragma unroll
    for (int k = 0; k < K; k++) {
        const int32_t t = tuples[(size_t)i * K + k];
        tk[k] = tris[t];
        ak[k] = attribs[t];
    }
    float x[2 * K];
#pragma unroll
    for (int j = 0; j < 2 * K; j++) x[j] = params[(size_t)i * 2 * K + j];
    int last = -1;
    const bool ok = palzilla_b200::solveConstraints<K>(x, p_beg, p_end[i], tk, ak, etas[i],
                                                      palzilla_b200::EventDescriptor::fromU32(events), maxIterations,
                                                      costTolerance, warmup, LastIteration{&last});
#pragma unroll
    for (int j = 0; j < 2 * K; j++) params[(size_t)i * 2 * K + j] = x[j];
    if (converged) converged[i] = ok ? 1 : 0;
    if (iters) iters[i] = last;
}

template <int K>
cudaError_t launch(uint32_t events, float3 p_beg, const int32_t* tuples, const float3* p_end, const float* etas,
                   uint32_t n, const pz_triangle* tris, const pz_triangle_attrib* attribs, uint32_t nTris,
                   int maxIterations, float tol, int warmup, float* params, uint8_t* conv, int32_t* iters,
                   cudaStream_t s)
{
    k_solve_constraints<K><<<(n + 255) / 256, 256, 0, s>>>(events, p_beg, tuples, p_end, etas, n, tris, attribs, nTris,
                                                           maxIterations, tol, warmup, params, conv, iters);
    return cudaGetLastError();
}

}  // namespace
}  // namespace pz

using namespace pz;

extern "C" int pz_solve_constraints(int K, uint32_t events, pz_float3 p_beg, const int32_t* tuples_dev,
                                    const pz_float3* p_end_dev, const float* etas_dev, uint32_t n,
                                    const pz_triangle* triangles_dev, const pz_triangle_attrib* attribs_dev,
                                    uint32_t n_triangles, int max_iterations, float cost_tolerance, int early_term_warmup, float* params_dev,
                                    uint8_t* converged_dev, int32_t* iters_dev, pz_stream_t stream)
{
    if (K < 1 || K > 4) return fail(PZ_ERR_INVALID_ARGUMENT, "pz_solve_constraints: K must be 1..4 (got %d)", K);
    if ((int)(events >> 24) != K)
        return fail(PZ_ERR_INVALID_ARGUMENT, "pz_solve_constraints: event descriptor size %u != K %d", events >> 24, K);
    if (max_iterations < 0) return fail(PZ_ERR_INVALID_ARGUMENT, "pz_solve_constraints: negative max_iterations");
    if (n == 0) {
        clear_error();
        return PZ_OK;
    }
    if (!tuples_dev || !p_end_dev || !etas_dev || !triangles_dev || !attribs_dev || !params_dev)
        return fail(PZ_ERR_INVALID_ARGUMENT, "pz_solve_constraints: null buffer");
    const float3 pb = make_float3(p_beg.x, p_beg.y, p_beg.z);
    const float3* pe = reinterpret_cast<const float3*>(p_end_dev);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    cudaError_t e = cudaErrorInvalidValue;
    switch (K) {
        case 1: e = launch<1>(events, pb, tuples_dev, pe, etas_dev, n, triangles_dev, attribs_dev, n_triangles, max_iterations,
                              cost_tolerance, early_term_warmup, params_dev, converged_dev, iters_dev, s); break;
        case 2: e = launch<2>(events, pb, tuples_dev, pe, etas_dev, n, triangles_dev, attribs_dev, n_triangles, max_iterations,
                              cost_tolerance, early_term_warmup, params_dev, converged_dev, iters_dev, s); break;
        case 3: e = launch<3>(events, pb, tuples_dev, pe, etas_dev, n, triangles_dev, attribs_dev, n_triangles, max_iterations,
                              cost_tolerance, early_term_warmup, params_dev, converged_dev, iters_dev, s); break;
        case 4: e = launch<4>(events, pb, tuples_dev, pe, etas_dev, n, triangles_dev, attribs_dev, n_triangles, max_iterations,
                              cost_tolerance, early_term_warmup, params_dev, converged_dev, iters_dev, s); break;
    }
    return done(e, "pz_solve_constraints");
}
