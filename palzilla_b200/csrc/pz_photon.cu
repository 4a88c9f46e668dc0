// pz_photon.cu -- photon pass: trace photons from the point light through specular
// triangles and gather the landing paths into the PathCache (photonTrace,
// main_gpu.cu:56-211; PathCache::store, pk.h:291-349).
//
// Photon identity is (triangle, j): photon j of triangle t uses Sobol index j with
// scramble seeds (iteration, t, 789) for the position and (iteration, t, 178) for
// eta, and (j, depth, t, iteration) for the Fresnel choice at each bounce -- exactly
// the reference's streams -- so the traced paths are bit-exact with the oracle (this
// unit is compiled with -fmad=false).  One thread per photon: the grid covers
// n_triangles x photons_per_triangle photons (the reference's 256-thread block per
// triangle is the photons_per_triangle = 256 case).  Diffuse and back-facing
// emitters retire at once, as in the reference.
//
// PathCache stores (PathCache::store, pk.h:291-349) are made by the whole warp at the
// end: each landed photon's 8 cell probes are spread over the warp's lanes, the photon's
// tuple passed through shared memory, so a warp with few landings does not run 8 probes
// in a row on one lane; a probe chain longer than a few slots is then walked by the whole
// warp, 32 slots per read.  Which photon's barycentrics fill a new slot is decided by the
// CAS race, as in the reference.
#include "pz_cache.cuh"
#include "pz_optics.cuh"
#include "pz_photon.cuh"
#include "pz_trace.cuh"

namespace pz {

constexpr int kPhotonDepth = 4;  // PHOTON_TRACE_MAX_DEPTH, pk.h:33
constexpr int kPhotonBlock = 256;

// slots a lane probes on its own before the warp walks the rest of its chain (sphere
// frame: 4 -> 7.27 ms, 8 -> 7.00, 16 -> 6.83, no warp walk -> 8.28)
#ifndef PZ_CACHE_SHORT_PROBE
#define PZ_CACHE_SHORT_PROBE 16
#endif

#ifndef PZ_PHOTON_MIN_BLOCKS
#define PZ_PHOTON_MIN_BLOCKS 1
#endif

__global__ void __launch_bounds__(kPhotonBlock, PZ_PHOTON_MIN_BLOCKS) k_photon(const Node* __restrict__ nodes, const uint32_t* __restrict__ rootPtr,
                                                const Tri* __restrict__ tris, const Attrib* __restrict__ attribs,
                                                uint32_t nTris, uint32_t photonsPerTri, float3 p_light, float eta_min,
                                                float eta_max, int iteration, float minThroughput, CacheView cache,
                                                PhotonRecord* __restrict__ records)
{
    const uint64_t gid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t iTri = (uint32_t)(gid / photonsPerTri);
    const uint32_t j = (uint32_t)(gid % photonsPerTri);
    const bool live = iTri < nTris;  // every lane reaches the warp's stores below
    bool landed = false;
    float3 p_land = mk3(0.f, 0.f, 0.f);
    uint32_t ev_land = 0;
    int4 t_land = make_int4(0, 0, 0, 0);
    float4 b0 = make_float4(0.f, 0.f, 0.f, 0.f), b1 = b0;
    PhotonRecord rec;
    rec.ev = 0;
    bool emitted = false;
    const uint32_t root = __ldg(rootPtr);

    const int32_t mat0 = live ? __ldg(&attribs[iTri].material) : kDiffuse;
    if (mat0 != kDiffuse) {
        float3 v0, v1, v2;
        load_tri(tris, iTri, v0, v1, v2);
        float3 ng0 = cross(v1 - v0, v2 - v0);
        const float* an = reinterpret_cast<const float*>(attribs + iTri) + 1;
        float3 ns0 = mk3(__ldg(an + 0), __ldg(an + 1), __ldg(an + 2));
        ng0 = ng0 * dot(ng0, ns0);
        if (!(dot(ng0, p_light - v0) < 0.0f)) {
            float2 prm;
            sobol2d(&prm.x, &prm.y, j, (uint32_t)iteration, iTri, 789u);
            prm = square2triangle(prm);
            float2 er;
            sobol2d(&er.x, &er.y, j, (uint32_t)iteration, iTri, 178u);
            const float eta = lerpf(eta_min, eta_max, er.x);
            const float3 p = v0 + (v1 - v0) * prm.x + (v2 - v0) * prm.y;
            float3 ro = p_light, rd = p - p_light;
            uint32_t ev = 0;
            int K = 0;
            bool admissible = false;
            float throughput = 1.0f;
            float3 p_final = mk3(0.f, 0.f, 0.f);
            int triIdx[kPhotonDepth] = {0, 0, 0, 0};
            float params[2 * kPhotonDepth] = {0, 0, 0, 0, 0, 0, 0, 0};
            for (int d = 0; d < kPhotonDepth + 1; d++) {
                Hit hit = make_miss();
                closest_hit(hit, nodes, tris, root, ro, rd, &cache.h->status);
                if (hit.t == kFltMax) break;
                const Attrib* A = attribs + hit.tri;
                const int32_t m = __ldg(&A->material);
                const float* sn = reinterpret_cast<const float*>(A) + 1;
                const float3 n0 = mk3(__ldg(sn + 0), __ldg(sn + 1), __ldg(sn + 2));
                const float3 n1 = mk3(__ldg(sn + 3), __ldg(sn + 4), __ldg(sn + 5));
                const float3 n2 = mk3(__ldg(sn + 6), __ldg(sn + 7), __ldg(sn + 8));
                const float3 p_hit = ro + rd * hit.t;
                const float3 ns = n0 + (n1 - n0) * hit.u + (n2 - n0) * hit.v;
                if (m == kDiffuse) {
                    if (d == 0) break;
                    admissible = true;
                    p_final = p_hit;
                    break;
                }
                if (d == kPhotonDepth) break;
                const float3 wi = -rd;
                triIdx[d] = (int)hit.tri;
                params[2 * d] = hit.u;
                params[2 * d + 1] = hit.v;
                float2 rnd;
                sobol2d(&rnd.x, &rnd.y, j, (uint32_t)d, iTri, (uint32_t)iteration);
                const float reflectance = fresnel_exact_norm_free(wi, ns, eta);
                const bool isT = (m == kDielectric) && !(rnd.x < reflectance);
                if (isT) ev |= 1u << K;
                K++;
                float sign = 1.0f;
                float3 wo;
                if (!isT) {
                    wo = reflection(wi, ns);
                    if (m == kDielectric) throughput *= reflectance;
                } else {
                    if (!refraction_norm_free(&wo, wi, ns, eta)) break;
                    sign = -1.0f;
                    throughput *= 1.0f - reflectance;
                }
                if (0.0f < dot(hit.ng, wi) * dot(hit.ng, wo) * sign) {
                    const float3 od = normalize(hit.ng * dot(hit.ng, wo));
                    ro = p_hit + od * ray_offset_scale(p_hit);
                    rd = wo;
                    continue;
                }
                break;
            }
            if (admissible && minThroughput < throughput) {
                ev |= (uint32_t)K << 24;
                emitted = true;
                if (cache.hash) {
                    landed = true;
                    p_land = p_final;
                    ev_land = ev;
                    t_land = make_int4(triIdx[0], K > 1 ? triIdx[1] : 0, K > 2 ? triIdx[2] : 0, K > 3 ? triIdx[3] : 0);
                    float q[8];
                    for (int d = 0; d < 8; d++) q[d] = d < 2 * K ? params[d] : 0.0f;
                    b0 = make_float4(q[0], q[1], q[2], q[3]);
                    b1 = make_float4(q[4], q[5], q[6], q[7]);
                }
                if (records) {
                    rec.ev = ev;
                    for (int d = 0; d < 4; d++) rec.tris[d] = triIdx[d];
                    for (int d = 0; d < 8; d++) rec.params[d] = params[d];
                    rec.p[0] = p_final.x;
                    rec.p[1] = p_final.y;
                    rec.p[2] = p_final.z;
                }
            }
        }
    }
    // the warp's landed photons, packed to the front of the warp's shared slots: landing
    // point with the path hash in w, event descriptor, triangles, barycentrics
    __shared__ float4 shPos[kPhotonBlock];
    __shared__ uint32_t shEv[kPhotonBlock];
    __shared__ int4 shTris[kPhotonBlock];
    __shared__ float4 shBary[2 * kPhotonBlock];
    __syncwarp();
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t landMask = __ballot_sync(0xffffffffu, landed);
    const int nLand = __popc(landMask);
    const int warpBase = (int)(threadIdx.x & ~31u);
    if (landed) {
        const int r = warpBase + __popc(landMask & ((1u << lane) - 1u));
        const int tl[4] = {t_land.x, t_land.y, t_land.z, t_land.w};
        shPos[r] = make_float4(p_land.x, p_land.y, p_land.z, __uint_as_float(path_hash(ev_land, tl)));
        shEv[r] = ev_land;
        shTris[r] = t_land;
        shBary[2 * r] = b0;
        shBary[2 * r + 1] = b1;
    }
    __syncwarp();
    // Each lane probes its cell for up to PZ_CACHE_SHORT_PROBE slots; the chains left over
    // are walked by the whole warp, one at a time, 32 slots per read: the first slot that
    // holds the path or reads empty decides, as in the one-slot-at-a-time walk.
    const int nTask = 8 * nLand;
    const uint32_t mask = cache.capacity - 1u;
    for (int round = 0; round < ((nTask + 31) >> 5); round++) {
        const int task = (round << 5) + (int)lane;
        const int src = warpBase + (min(task, nTask - 1) >> 3);
        bool pending = task < nTask;
        uint32_t hP = 0, hp = 0, i = 0, off = 0;
        if (pending) {
            const float4 pw = shPos[src];
            hP = cache_cell_hash(cache, mk3(pw.x, pw.y, pw.z), task & 7);
            hp = __float_as_uint(pw.w);
            i = hP & mask;
            pending = cache_probe(cache, hP, hp, shEv[src], shTris[src], shBary[2 * src], shBary[2 * src + 1], i, off,
                                  PZ_CACHE_SHORT_PROBE);
        }
        uint32_t longMask = __ballot_sync(0xffffffffu, pending);
        while (longMask != 0u) {
            const int leader = __ffs(longMask) - 1;
            const uint32_t lhp = __shfl_sync(0xffffffffu, hp, leader);
            const uint32_t li = __shfl_sync(0xffffffffu, i, leader);
            const uint32_t loff = __shfl_sync(0xffffffffu, off, leader);
            const bool inRange = loff + lane < kMaxProbe;
            const uint32_t seen = inRange ? __ldcg(cache.hash + ((li + lane) & mask)) : 0u;
            const uint32_t hitMask = __ballot_sync(0xffffffffu, inRange && seen == lhp);
            const uint32_t stopMask = __ballot_sync(0xffffffffu, inRange && (seen == lhp || seen == 0u));
            if ((int)lane == leader) {
                if (stopMask == 0u) {
                    i = (li + 32u) & mask;
                    off = loff + 32u;
                } else {
                    const uint32_t f = (uint32_t)(__ffs(stopMask) - 1);
                    const uint32_t slot = (li + f) & mask;
                    if ((hitMask >> f) & 1u) {
                        pending = false;
                    } else {
                        const uint32_t old = atomicCAS(cache.hash + slot, 0u, hp);
                        if (old == 0u) {
                            cache_fill_slot(cache, slot, hP, shEv[src], shTris[src], shBary[2 * src], shBary[2 * src + 1]);
                            pending = false;
                        } else if (old == hp) {
                            pending = false;
                        } else {
                            i = (slot + 1u) & mask;
                            off = loff + f + 1u;
                        }
                    }
                }
                if (pending && off >= kMaxProbe) {
                    raise_error(&cache.h->status, kErrCapacity);
                    pending = false;
                }
            }
            longMask = __ballot_sync(0xffffffffu, pending);
        }
    }
    if (!live) return;
    if (records) {
        if (!emitted) {
            for (int d = 0; d < 4; d++) rec.tris[d] = 0;
            for (int d = 0; d < 8; d++) rec.params[d] = 0.0f;
            rec.p[0] = rec.p[1] = rec.p[2] = 0.0f;
        }
        records[gid] = rec;
    }
}

cudaError_t launch_photons(const Node* nodes, const uint32_t* root, const Tri* tris, const Attrib* attribs,
                           uint32_t nTris, uint32_t photonsPerTri, float3 p_light, float eta_min, float eta_max,
                           int iteration, float minThroughput, const CacheView& cache, PhotonRecord* records,
                           cudaStream_t s)
{
    const uint64_t total = (uint64_t)nTris * photonsPerTri;
    if (total == 0) return cudaSuccess;
    const uint64_t blocks = (total + 255) / 256;
    k_photon<<<(unsigned)blocks, kPhotonBlock, 0, s>>>(nodes, root, tris, attribs, nTris, photonsPerTri, p_light, eta_min,
                                              eta_max, iteration, minThroughput, cache, records);
    return cudaGetLastError();
}

}  // namespace pz
