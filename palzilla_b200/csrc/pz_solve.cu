// pz_solve.cu -- the plain per-tuple specular solve and the resolve (tone map) kernels.
//
// k_solve_plain<K, kBinned>: solveSpecularPath<K> (main_gpu.cu:418-486): one thread per
// work item -- (pixel, cached tuple) with the pixel's sampled wavelength, or, in binned
// mode, (pixel, cached tuple, wavelength bin) -- starting from the photon's
// barycentrics: Newton solve, admissibility + visibility, dAdw, clamped contribution
// accumulated with atomics (RGB in reference mode, one spectral bin in binned mode).
// This is the structure the batched persistent solver is measured against.
//
// The unit is compiled twice: as is (FMA contraction on: the performance baseline) and
// with -DPZ_SOLVE_EXACT -fmad=false, which gives results bit-compatible with the CPU
// oracle for the parity tests.
#include "pz_frame.cuh"
#include "pz_solve.cuh"
#include "pz_solver.cuh"

#ifdef PZ_SOLVE_EXACT
#define PZ_SOLVE_NS exact
#define PZ_SOLVE_LAUNCH launch_solve_plain_exact
#else
#define PZ_SOLVE_NS fast
#define PZ_SOLVE_LAUNCH launch_solve_plain
#endif

namespace pz {
namespace PZ_SOLVE_NS {

using solver::V3;

PZ_D void count_stats(unsigned long long* stats, bool converged, bool contributing)
{
    // warp-aggregated counters: items, converged, contributing
    const uint32_t active = __activemask();
    const uint32_t c = __ballot_sync(active, converged), k = __ballot_sync(active, contributing);
    if ((threadIdx.x & 31) == __ffs(active) - 1) {
        atomicAdd(stats + 0, (unsigned long long)__popc(active));
        atomicAdd(stats + 1, (unsigned long long)__popc(c));
        atomicAdd(stats + 2, (unsigned long long)__popc(k));
    }
}

template <int K, bool kBinned>
__global__ void __launch_bounds__(256) k_solve_plain(SolveArgs a)
{
    const uint64_t item = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t nb = kBinned ? (uint32_t)a.nBins : 1u;
    const uint64_t pathIdx = item / nb;
    const uint32_t bin = (uint32_t)(item % nb);
    if (pathIdx >= a.nPaths) return;
    const SpecularPath sp = a.paths[pathIdx];
    const FirstDiffuse fd = a.fds[sp.pixel];
    const int4 ti = a.cache.tris[sp.cacheIndex];
    const float4 p0 = a.cache.params[2 * sp.cacheIndex], p1 = a.cache.params[2 * sp.cacheIndex + 1];
    const int idx[4] = {ti.x, ti.y, ti.z, ti.w};
    solver::Chain<K> ch;
    solver::load_chain<K>(ch, a.tris, a.attribs, idx);
    const float pp[8] = {p0.x, p0.y, p0.z, p0.w, p1.x, p1.y, p1.z, p1.w};
    float prm[2 * K];
#pragma unroll
    for (int i = 0; i < 2 * K; i++) prm[i] = pp[i];
    const float eta = kBinned ? a.etas[bin] : a.cauchyA + a.cauchyB / (fd.lambda * fd.lambda);
    const V3<float> L = solver::v3f<float>(a.p_light), p = solver::v3f<float>(fd.p);
    const uint32_t root = __ldg(a.root);
    bool conv = solver::solve_constraints<float, K>(prm, L, p, ch, eta, a.events, a.maxIterations, a.costTolerance,
                                                    a.earlyTermWarmUp);
    bool contributing = false;
    if (conv && a.roots) {
        float* r = a.roots + (pathIdx * nb + bin) * 8;
#pragma unroll
        for (int i = 0; i < 2 * K; i++) r[i] = prm[i];
    }
    if (conv) {
        const float thr = solver::contributable_throughput<float, K>(prm, L, p, ch, a.events, a.nodes, a.tris, root, eta);
        if (0.0f < thr) {
            contributing = true;
            const V3<float> v0 = solver::vertex<float, K>(ch, prm, 0);
            const float dAdwValue = solver::dadw<float, K>(L, v0 - L, p, ch, a.events, eta);
            const V3<float> vl = solver::vertex<float, K>(ch, prm, K - 1);
            const float cosv = fmaxf(solver::vdot(solver::vnormalize(vl - p), solver::v3f<float>(fd.ng)), 0.0f);
            float contrib = thr * a.lightIntensity / dAdwValue * cosv;
            contrib = fminf(contrib, a.radianceClamp);
            if (kBinned) {
                atomicAdd(a.spectral + (size_t)sp.pixel * nb + bin, contrib);
            } else {
                const float p_lambda = cmf_y_pdf(fd.lambda);
                const float3 Lr = (fd.R / kPi) * lambda_to_srgb(fd.lambda) * contrib / p_lambda;
                atomicAdd(&a.accum[sp.pixel].x, Lr.x);
                atomicAdd(&a.accum[sp.pixel].y, Lr.y);
                atomicAdd(&a.accum[sp.pixel].z, Lr.z);
            }
        }
    }
    if (a.stats) count_stats(a.stats, conv, contributing);
}

template <int K, bool kB>
static cudaError_t launch_k(const SolveArgs& a, cudaStream_t s)
{
    const uint64_t items = a.nPaths * (uint64_t)(kB ? a.nBins : 1);
    if (items == 0) return cudaSuccess;
    k_solve_plain<K, kB><<<(unsigned)((items + 255) / 256), 256, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace PZ_SOLVE_NS

cudaError_t PZ_SOLVE_LAUNCH(int K, bool binned, const SolveArgs& a, cudaStream_t s)
{
    using namespace PZ_SOLVE_NS;
    switch (K * 2 + (binned ? 1 : 0)) {
        case 2: return launch_k<1, false>(a, s);
        case 3: return launch_k<1, true>(a, s);
        case 4: return launch_k<2, false>(a, s);
        case 5: return launch_k<2, true>(a, s);
        case 6: return launch_k<3, false>(a, s);
        case 7: return launch_k<3, true>(a, s);
        case 8: return launch_k<4, false>(a, s);
        case 9: return launch_k<4, true>(a, s);
    }
    return cudaErrorInvalidValue;
}

#ifndef PZ_SOLVE_EXACT
// ---------------------------------------------------------------- resolve
PZ_D float srgb_oetf(float r)  // pk.h:1023-1031
{
    r = fmaxf(r, 0.0f);
    if (r <= 0.003130f) return 12.92f * r;
    return 1.055f * powf(r, 1.0f / 2.4f) - 0.055f;
}
PZ_D uint32_t pack_rgba(float r, float g, float b)  // packRGBA, main_gpu.cu:9-14
{
    const int ir = max(0, min(__float2int_rz(r * 255.0f + 0.5f), 255));
    const int ig = max(0, min(__float2int_rz(g * 255.0f + 0.5f), 255));
    const int ib = max(0, min(__float2int_rz(b * 255.0f + 0.5f), 255));
    return 0xFF000000u | ((uint32_t)ib << 16) | ((uint32_t)ig << 8) | (uint32_t)ir;
}

__global__ void k_pack(uint32_t* __restrict__ pixels, const float4* __restrict__ accum, int n)  // main_gpu.cu:499-513
{
    const int i = blockIdx.x * 256 + threadIdx.x;
    if (i >= n) return;
    const float4 a = accum[i];
    pixels[i] = pack_rgba(srgb_oetf(a.x / a.w), srgb_oetf(a.y / a.w), srgb_oetf(a.z / a.w));
}

// Spectral image -> linear sRGB: (albedo / pi) * sum_b S_b * srgb(lambda_b) * dlambda (the
// quadrature of the reference's Monte Carlo estimate L = (R/pi) srgb(l) contrib / p(l)).
__global__ void k_resolve_spectral(float4* __restrict__ rgb, uint32_t* __restrict__ pixels,
                                   const float* __restrict__ spectral, int n, int nBins, float lambdaMin,
                                   float lambdaMax, float3 albedo)
{
    const int i = blockIdx.x * 256 + threadIdx.x;
    if (i >= n) return;
    const float w = (lambdaMax - lambdaMin) / (float)nBins;
    float3 c = mk3(0.f, 0.f, 0.f);
    for (int b = 0; b < nBins; b++) {
        const float lam = lambdaMin + ((float)b + 0.5f) * w;
        c = c + lambda_to_srgb(lam) * (spectral[(size_t)i * nBins + b] * w);
    }
    c = (albedo / kPi) * c;
    if (rgb) rgb[i] = make_float4(c.x, c.y, c.z, 1.0f);
    if (pixels) pixels[i] = pack_rgba(srgb_oetf(c.x), srgb_oetf(c.y), srgb_oetf(c.z));
}

cudaError_t launch_pack(uint32_t* pixels, const float4* accum, int n, cudaStream_t s)
{
    if (n <= 0) return cudaSuccess;
    k_pack<<<(n + 255) / 256, 256, 0, s>>>(pixels, accum, n);
    return cudaGetLastError();
}

cudaError_t launch_resolve_spectral(float4* rgb, uint32_t* pixels, const float* spectral, int n, int nBins,
                                    float lambdaMin, float lambdaMax, float3 albedo, cudaStream_t s)
{
    if (n <= 0) return cudaSuccess;
    k_resolve_spectral<<<(n + 255) / 256, 256, 0, s>>>(rgb, pixels, spectral, n, nBins, lambdaMin, lambdaMax, albedo);
    return cudaGetLastError();
}

#endif  // PZ_SOLVE_EXACT

}  // namespace pz
