// pz_solve.cuh -- specular solve interfaces.
#pragma once
#include "pz_frame.cuh"

namespace pz {

struct SolveArgs {
    float4* accum;             // reference mode: RGB accumulator (w = sample count)
    float* spectral;           // binned mode: [pixel][bin]
    const float* etas;         // binned mode: eta per bin
    int nBins;
    const SpecularPath* paths;
    uint64_t nPaths;
    const FirstDiffuse* fds;
    const Node* nodes;
    const uint32_t* root;
    const Tri* tris;
    const Attrib* attribs;
    float3 p_light;
    float lightIntensity;
    float radianceClamp;
    CacheView cache;
    uint32_t events;
    float cauchyA, cauchyB;
    int maxIterations;         // 32 (main_gpu.cu:456)
    float costTolerance;       // 1e-10
    int earlyTermWarmUp;       // 1
    unsigned long long* stats; // [solves, converged, contributing] or null
    float* roots;              // converged roots, 8 floats per (item, bin), or null
};

cudaError_t launch_solve_plain(int K, bool binned, const SolveArgs& a, cudaStream_t s);
// the same kernels without FMA contraction (bit-compatible with the CPU oracle)
cudaError_t launch_solve_plain_exact(int K, bool binned, const SolveArgs& a, cudaStream_t s);
cudaError_t launch_pack(uint32_t* pixels, const float4* accum, int n, cudaStream_t s);
cudaError_t launch_resolve_spectral(float4* rgb, uint32_t* pixels, const float* spectral, int n, int nBins,
                                    float lambdaMin, float lambdaMax, float3 albedo, cudaStream_t s);

}  // namespace pz
