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
struct Tex {  // Texture8RGBX, pk.h:1075-1098 (texels == null: the constant albedo)
    const uint8_t* texels;
    uint32_t w, h;
};

// Texture8RGBX::samplePoint (pk.h:1083-1095): repeat wrapping, nearest texel, gamma 2.2.
PZ_D float3 sample_point(const Tex& t, float u, float v)
{
    u = u - floorf(u);
    v = v - floorf(v);
    const int ix = (int)fminf(u * (float)t.w, (float)t.w - 1.0f);
    const int iy = (int)fminf(v * (float)t.h, (float)t.h - 1.0f);
    const uint32_t i = (uint32_t)ix + t.w * (uint32_t)iy;
    const uchar4 c = __ldg(reinterpret_cast<const uchar4*>(t.texels) + i);
    return mk3(powf((float)c.x / 255.0f, 2.2f), powf((float)c.y / 255.0f, 2.2f), powf((float)c.z / 255.0f, 2.2f));
}

cudaError_t launch_primary(float4* accum, FirstDiffuse* fds, int W, int H, const RayGen& g, const Lens& lens,
                           const Node* nodes, const uint32_t* root, const Tri* tris, const Attrib* attribs,
                           float3 p_light, float lightIntensity, float radianceClamp, float cauchyA, float cauchyB,
                           float3 albedo, const Tex& tex, int iteration, uint32_t* status, cudaStream_t s);
cudaError_t launch_lookup(uint32_t ev, SpecularPath* paths, unsigned long long* indexed, uint32_t* counter,
                          uint32_t capacity, const FirstDiffuse* fds, int nPixels, const CacheView& cache,
                          cudaStream_t s);
cudaError_t launch_reorder(const unsigned long long* indexed, SpecularPath* dst, const SpecularPath* src, uint32_t n,
                           cudaStream_t s);

}  // namespace pz
