// pz_frame.cuh -- eye pass / work-list interfaces and the per-frame records.
#pragma once
#include "pz_cache.cuh"

namespace pz {

struct FirstDiffuse {  // pk.h:80-86 (40 B)
    float3 p;
    float3 ng;
    float3 R;
    float lambda;
};
static_assert(sizeof(FirstDiffuse) == 40, "FirstDiffuse layout");

struct SpecularPath {  // pk.h:1102-1106
    int pixel;
    int cacheIndex;
};

struct RayGen {  // RayGenerator, camera.h:4-41
    float3 origin, right, up;
};
struct Lens {  // LensParams, pk.h:1035-1040 (R <= 0 disables the lens)
    float distance, thickness, R;
};

cudaError_t launch_primary(float4* accum, FirstDiffuse* fds, int W, int H, const RayGen& g, const Lens& lens,
                           const Node* nodes, const uint32_t* root, const Tri* tris, const Attrib* attribs,
                           float3 p_light, float lightIntensity, float radianceClamp, float cauchyA, float cauchyB,
                           float3 albedo, int iteration, uint32_t* status, cudaStream_t s);
cudaError_t launch_lookup(uint32_t ev, SpecularPath* paths, unsigned long long* indexed, uint32_t* counter,
                          uint32_t capacity, const FirstDiffuse* fds, int nPixels, const CacheView& cache,
                          cudaStream_t s);
cudaError_t launch_reorder(const unsigned long long* indexed, SpecularPath* dst, const SpecularPath* src, uint32_t n,
                           cudaStream_t s);

}  // namespace pz
