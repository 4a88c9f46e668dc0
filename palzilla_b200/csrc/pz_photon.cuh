// pz_photon.cuh -- photon pass interface (see pz_photon.cu).
#pragma once
#include "pz_cache.cuh"

namespace pz {

// 64-byte debug record of one photon; ev == 0 when the photon produced no path.
struct PhotonRecord {
    uint32_t ev;
    int32_t tris[4];
    float params[8];
    float p[3];
};
static_assert(sizeof(PhotonRecord) == 64, "record layout");

cudaError_t launch_photons(const Node* nodes, const uint32_t* root, const Tri* tris, const Attrib* attribs,
                           uint32_t nTris, uint32_t photonsPerTri, float3 p_light, float eta_min, float eta_max,
                           int iteration, float minThroughput, const CacheView& cache, PhotonRecord* records,
                           cudaStream_t s);

}  // namespace pz
