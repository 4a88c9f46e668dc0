// pz_oracle_capi.cpp -- TEST INFRASTRUCTURE ONLY: flat C entry points over the
// CPU restatement in pz_oracle.hpp, loaded by tests/ (ctypes) and by bench.py's
// CPU-baseline leg.  Nothing in the product links or loads this library.
#include "pz_oracle.hpp"
#include "pz_oracle_subdiv.hpp"

#include <omp.h>

#include <array>
#include <atomic>
#include <tuple>
#include <cstdio>

using namespace pzo;

namespace {
inline F3 ld3(const float* p) { return mk(p[0], p[1], p[2]); }
inline void st3(float* p, F3 v) { p[0] = v.x; p[1] = v.y; p[2] = v.z; }
}  // namespace

extern "C" {

int pzo_version(void) { return 1; }
int pzo_max_threads(void) { return omp_get_max_threads(); }
void pzo_set_threads(int n) { if (n > 0) omp_set_num_threads(n); }

// ---------------------------------------------------------------- LBVH
void pzo_scene_aabb(const Triangle* tris, int n, float* out6)
{
    AABB b = scene_aabb(tris, n);
    st3(out6, b.lower);
    st3(out6 + 3, b.upper);
}

void pzo_morton_keys(const Triangle* tris, int n, uint32_t opt, const float* aabb6, uint32_t* keys)
{
    AABB b{ld3(aabb6), ld3(aabb6 + 3)};
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; i++) keys[i] = morton_key(tris[i], b, opt);
}

// Stable LSD sort of 64-bit elements on key bits [startBit, endBit): the order the
// onesweep sort (tinyhiponesweep.h:602-668) produces.
// Digit passes cover whole 8-bit digits (tinyhiponesweep.h:606, :93-94), so the key
// field is rounded up to a multiple of 8 bits above startBit.
static inline int digit_end(int startBit, int endBit) { return startBit + 8 * ((endBit - startBit + 7) / 8); }
void pzo_stable_sort_u64(uint64_t* keys, uint32_t n, int startBit, int endBit)
{
    endBit = digit_end(startBit, endBit);
    uint64_t mask = (endBit - startBit >= 64) ? ~0ull : (((1ull << (endBit - startBit)) - 1ull) << startBit);
    std::stable_sort(keys, keys + n, [mask](uint64_t a, uint64_t b) { return (a & mask) < (b & mask); });
}
void pzo_stable_sort_u32(uint32_t* keys, uint32_t n, int startBit, int endBit)
{
    endBit = digit_end(startBit, endBit);
    if (endBit > 32) endBit = 32;
    uint32_t mask = (endBit - startBit >= 32) ? ~0u : (((1u << (endBit - startBit)) - 1u) << startBit);
    std::stable_sort(keys, keys + n, [mask](uint32_t a, uint32_t b) { return (a & mask) < (b & mask); });
}
// Stable key/value sort (keys u32 or u64 by width, values u32).
void pzo_stable_sort_kv(void* keys, uint32_t* values, uint32_t n, int keyBytes, int startBit, int endBit)
{
    endBit = digit_end(startBit, endBit);
    if (endBit > 8 * keyBytes) endBit = 8 * keyBytes;
    std::vector<uint32_t> perm(n);
    for (uint32_t i = 0; i < n; i++) perm[i] = i;
    if (keyBytes == 8) {
        uint64_t* k = (uint64_t*)keys;
        uint64_t mask = (endBit - startBit >= 64) ? ~0ull : (((1ull << (endBit - startBit)) - 1ull) << startBit);
        std::stable_sort(perm.begin(), perm.end(), [&](uint32_t a, uint32_t b) { return (k[a] & mask) < (k[b] & mask); });
        std::vector<uint64_t> tk(k, k + n);
        std::vector<uint32_t> tv(values, values + n);
        for (uint32_t i = 0; i < n; i++) { k[i] = tk[perm[i]]; values[i] = tv[perm[i]]; }
    } else {
        uint32_t* k = (uint32_t*)keys;
        uint32_t mask = (endBit - startBit >= 32) ? ~0u : (((1u << (endBit - startBit)) - 1u) << startBit);
        std::stable_sort(perm.begin(), perm.end(), [&](uint32_t a, uint32_t b) { return (k[a] & mask) < (k[b] & mask); });
        std::vector<uint32_t> tk(k, k + n);
        std::vector<uint32_t> tv(values, values + n);
        for (uint32_t i = 0; i < n; i++) { k[i] = tk[perm[i]]; values[i] = tv[perm[i]]; }
    }
}

// Full builder: outputs nodes (n-1), root, the sorted (morton,index) pairs and deltas.
int pzo_build_bvh(const Triangle* tris, int n, uint32_t opt, InternalNode* nodes_out, uint32_t* root_out,
                  uint64_t* sorted_out, uint8_t* deltas_out, float* aabb_out6)
{
    LBVH b;
    build_bvh(b, tris, n, opt);
    if (n > 1) std::memcpy(nodes_out, b.nodes.data(), sizeof(InternalNode) * (size_t)(n - 1));
    *root_out = b.root;
    if (sorted_out)
        for (int i = 0; i < n; i++) sorted_out[i] = (uint64_t)b.sorted[i].morton | ((uint64_t)b.sorted[i].index << 32);
    if (deltas_out && n > 1) std::memcpy(deltas_out, b.deltas.data(), (size_t)(n - 1));
    if (aabb_out6) { st3(aabb_out6, b.scene.lower); st3(aabb_out6 + 3, b.scene.upper); }
    return 0;
}

int pzo_validate_lbvh(const InternalNode* nodes, uint32_t root, const uint8_t* deltas)
{
    return validate_lbvh(root, nodes, deltas, 255) ? 1 : 0;
}

// ---------------------------------------------------------------- ray queries
// hits: t[n], uv[2n], tri[n], ng[3n]
void pzo_trace_closest(const InternalNode* nodes, uint32_t root, const Triangle* tris, int n, const float* ro,
                       const float* rd, float* t, float* uv, uint32_t* tri, float* ng)
{
#pragma omp parallel for schedule(dynamic, 256)
    for (int i = 0; i < n; i++) {
        Hit h;
        F3 o = ld3(ro + 3 * i), d = ld3(rd + 3 * i);
        intersect_stackfull(&h, nodes, tris, root, o, d, inv_rd(d));
        t[i] = h.t;
        uv[2 * i] = h.u;
        uv[2 * i + 1] = h.v;
        tri[i] = h.triangleIndex;
        st3(ng + 3 * i, h.ng);
    }
}
// any-hit with t_max (escape-link traversal); writes 1 if occluded before t_max
void pzo_trace_any(const InternalNode* nodes, uint32_t root, const Triangle* tris, int n, const float* ro,
                   const float* rd, const float* tmax, uint8_t* hit_out)
{
#pragma omp parallel for schedule(dynamic, 256)
    for (int i = 0; i < n; i++) {
        Hit h;
        h.t = tmax[i];
        F3 o = ld3(ro + 3 * i), d = ld3(rd + 3 * i);
        intersect_escape_link(&h, nodes, tris, root, o, d, inv_rd(d), true);
        hit_out[i] = h.t < tmax[i] ? 1 : 0;
    }
}

// ---------------------------------------------------------------- photons + cache
// Record layout (64 B): u32 ev, i32 tris[4], f32 params[8], f32 p_final[3].
struct PhotonRecordC { uint32_t ev; int32_t tris[4]; float params[8]; float p[3]; };
static_assert(sizeof(PhotonRecordC) == 64, "record layout");

// Traces photons_per_tri photons from every triangle (main_gpu.cu:56-211, one
// photon per thread of a PHOTON_BLOCK_SIZE block).  Records come out ordered by
// (triangle, photon).  Returns the record count (or -count if capacity ran out).
int64_t pzo_photon_trace(const InternalNode* nodes, uint32_t root, const Triangle* tris, const TriangleAttrib* attribs,
                         int nTris, const float* p_light, float eta_min, float eta_max, int iteration,
                         float minThroughput, int photonsPerTri, PhotonRecordC* out, int64_t capacity)
{
    F3 L = ld3(p_light);
    std::vector<std::vector<PhotonRecordC>> perTri(nTris);
#pragma omp parallel for schedule(dynamic, 16)
    for (int t = 0; t < nTris; t++) {
        for (int j = 0; j < photonsPerTri; j++) {
            PhotonRecord r;
            if (photon_trace_one(&r, nodes, root, tris, attribs, t, (uint32_t)j, L, eta_min, eta_max, iteration,
                                 minThroughput)) {
                PhotonRecordC c;
                c.ev = r.ev;
                std::memcpy(c.tris, r.tris, sizeof(c.tris));
                std::memcpy(c.params, r.params, sizeof(c.params));
                st3(c.p, r.p_final);
                perTri[t].push_back(c);
            }
        }
    }
    int64_t n = 0;
    bool overflow = false;
    for (int t = 0; t < nTris; t++)
        for (auto& c : perTri[t]) {
            if (n < capacity) out[n] = c;
            else overflow = true;
            n++;
        }
    return overflow ? -n : n;
}

// Inserts records in order into a fresh PathCache (pk.h:291-349).  Output arrays
// have `capacity` slots (tris 4 per slot, params 8 per slot).  Returns the count.
int64_t pzo_cache_build(const PhotonRecordC* recs, int64_t n, uint32_t capacity, float step, uint32_t* hashOfPath,
                        uint32_t* cellHash, uint32_t* events, int32_t* trisOut, float* paramsOut)
{
    PathCache c;
    c.init(capacity, step);
    for (int64_t i = 0; i < n; i++) c.store(ld3(recs[i].p), recs[i].tris, recs[i].params, recs[i].ev);
    std::memcpy(hashOfPath, c.hashOfPath.data(), sizeof(uint32_t) * capacity);
    std::memcpy(cellHash, c.cellHash.data(), sizeof(uint32_t) * capacity);
    std::memcpy(events, c.events.data(), sizeof(uint32_t) * capacity);
    std::memcpy(trisOut, c.tris.data(), sizeof(int32_t) * 4 * (size_t)capacity);
    std::memcpy(paramsOut, c.params.data(), sizeof(float) * 8 * (size_t)capacity);
    return c.count;
}

uint32_t pzo_path_hash(uint32_t ev, const int32_t* tris) { return PathCache::path_hash(ev, tris); }
uint32_t pzo_spacial_hash(const float* p, float step) { return spacial_hash(ld3(p), step); }

// lookupFlatten (main_gpu.cu:373-416) over a given cache: per valid pixel, the
// matching slot indices in probe order.  counts[n_pixels]; pairs written as
// (pixel, slot) in pixel order.  Returns the pair count (negative on overflow).
int64_t pzo_lookup_flatten(const uint32_t* hashOfPath, const uint32_t* cellHash, const uint32_t* events,
                           uint32_t capacity, float step, const float* p /*3 per pixel*/, const uint8_t* valid,
                           int nPixels, uint32_t ev, int32_t* counts, int32_t* pairs /*2 per pair*/, int64_t pairCap)
{
    PathCache c;
    c.capacity = capacity;
    c.step = step;
    c.hashOfPath.assign(hashOfPath, hashOfPath + capacity);
    c.cellHash.assign(cellHash, cellHash + capacity);
    c.events.assign(events, events + capacity);
    std::vector<std::vector<int32_t>> lists(nPixels);
#pragma omp parallel for schedule(dynamic, 64)
    for (int px = 0; px < nPixels; px++) {
        if (!valid[px]) continue;
        c.lookup(ld3(p + 3 * px), ev, [&](uint32_t i) { lists[px].push_back((int32_t)i); });
    }
    int64_t n = 0;
    for (int px = 0; px < nPixels; px++) {
        counts[px] = (int32_t)lists[px].size();
        for (int32_t s : lists[px]) {
            if (n < pairCap) { pairs[2 * n] = px; pairs[2 * n + 1] = s; }
            n++;
        }
    }
    return n > pairCap ? -n : n;
}

// ---------------------------------------------------------------- camera + eye pass
void pzo_lookat(const float* eye, const float* center, const float* up, float fovy, int w, int h, float* out9)
{
    RayGenerator g = lookat(ld3(eye), ld3(center), ld3(up), fovy, w, h);
    st3(out9, g.origin);
    st3(out9 + 3, g.right);
    st3(out9 + 6, g.up);
}

// Texture8RGBX::samplePoint (pk.h:1083-1095): repeat wrapping, nearest texel, each channel
// decoded as (c / 255)^2.2.
static F3 sample_point(const uint8_t* tex, int tw, int th, float u, float v)
{
    u = u - std::floor(u);
    v = v - std::floor(v);
    const int ix = (int)std::fmin(u * (float)tw, (float)tw - 1.0f);
    const int iy = (int)std::fmin(v * (float)th, (float)th - 1.0f);
    const uint8_t* c = tex + 4 * ((size_t)ix + (size_t)tw * iy);
    return mk(std::pow((float)c[0] / 255.0f, 2.2f), std::pow((float)c[1] / 255.0f, 2.2f),
              std::pow((float)c[2] / 255.0f, 2.2f));
}

// solvePrimary (main_gpu.cu:213-371): the thick lens applied only when lensR > 0, and the
// diffuse hit's albedo from the floor texture tex (RGBX, tw x th) sampled at its (x, z), or
// the constant albedo3 when tex is null.
// out: firstDiffuse as 10 floats per pixel {p, ng, R, lambda}; accum 4 floats per pixel (added).
void pzo_solve_primary(float* accum, float* firstDiffuse, int W, int H, const float* rayGen9, const float* lens3,
                       const InternalNode* nodes, uint32_t root, const Triangle* tris, const TriangleAttrib* attribs,
                       const float* p_light, float lightIntensity, float radianceClamp, float cauchyA, float cauchyB,
                       const float* albedo3, const uint8_t* tex, int tw, int th, int iteration)
{
    RayGenerator g{ld3(rayGen9), ld3(rayGen9 + 3), ld3(rayGen9 + 6)};
    F3 L = ld3(p_light);
    const F3 albedoConst = ld3(albedo3);
#pragma omp parallel for schedule(dynamic, 4)
    for (int yi = 0; yi < H; yi++) {
        for (int xi = 0; xi < W; xi++) {
            int pixel = xi + yi * W;
            float jx, jy;
            sobol2d(&jx, &jy, (uint32_t)iteration, (uint32_t)xi, (uint32_t)yi, 0u);
            F3 ro, rd;
            shoot(g, &ro, &rd, ((float)xi + jx) / (float)W, ((float)yi + jy) / (float)H);
            float lrx, lry;
            sobol2d(&lrx, &lry, (uint32_t)iteration, (uint32_t)xi, (uint32_t)yi, 1u);
            float lambda = cmf_y_sample(lrx);
            float p_lambda = cmf_y_pdf(lambda);
            float eta = cauchy(cauchyA, cauchyB, lambda);
            if (lens3[2] > 0.0f) {  // solveLens, pk.h:1042-1073
                F3 fwd = normalize(cross(g.up, g.right));
                float distance = lens3[0], thickness = lens3[1], R = lens3[2];
                F3 lensO = g.origin + fwd * distance;
                F3 c1 = lensO + fwd * (R - thickness * 0.5f);
                F3 c2 = lensO - fwd * (R - thickness * 0.5f);
                float t1, t1b;
                sph_intersect(&t1, &t1b, ro, rd, c1, R);
                if (!(t1 < 0.0f)) {
                    F3 hit1 = ro + rd * t1;
                    F3 wo = rd;
                    refraction_norm_free(&wo, -rd, hit1 - c1, eta);
                    rd = wo;
                    ro = hit1;
                    float t2, t2b;
                    sph_intersect(&t2, &t2b, ro, rd, c2, R);
                    F3 hit2 = ro + rd * t2;
                    if (refraction_norm_free(&wo, -rd, hit2 - c2, eta)) { rd = wo; ro = hit2; }
                }
            }
            bool hasDiffuse = false;
            Hit last;
            uint32_t dimLevel = 2;
            for (int d = 0; d < 32; d++) {
                Hit hit;
                intersect_stackfull(&hit, nodes, tris, root, ro, rd, inv_rd(rd));
                if (hit.t == kFltMax) { last = hit; break; }
                const TriangleAttrib& at = attribs[hit.triangleIndex];
                float rx, ry;
                sobol2d(&rx, &ry, (uint32_t)iteration, (uint32_t)xi, (uint32_t)yi, dimLevel++);
                if (at.material == kDiffuse) { hasDiffuse = true; last = hit; break; }
                F3 p_hit = ro + rd * hit.t;
                F3 ns = at.shadingNormals[0] + (at.shadingNormals[1] - at.shadingNormals[0]) * hit.u +
                        (at.shadingNormals[2] - at.shadingNormals[0]) * hit.v;
                F3 wi = -rd;
                bool isT = false;
                if (at.material == kDielectric) isT = !(rx < fresnel_exact_norm_free(wi, ns, eta));
                float sign = 1.0f;
                F3 wo;
                if (!isT) wo = reflection(wi, ns);
                else {
                    if (!refraction_norm_free(&wo, wi, ns, eta)) break;
                    sign = -1.0f;
                }
                if (0.0f < dot(hit.ng, wi) * dot(hit.ng, wo) * sign) {
                    F3 od = normalize(hit.ng * dot(hit.ng, wo));
                    ro = p_hit + od * ray_offset_scale(p_hit);
                    rd = wo;
                    continue;
                }
                break;
            }
            float* fd = firstDiffuse + 10 * (size_t)pixel;
            float* acc = accum + 4 * (size_t)pixel;
            if (!hasDiffuse) {
                acc[3] += 1.0f;
                fd[6] = fd[7] = fd[8] = 0.0f;
                continue;
            }
            F3 p = ro + rd * last.t;
            F3 n = normalize(last.ng);
            if (0.0f < dot(n, rd)) n = -n;
            F3 toL = L - p;
            float d2 = dot(toL, toL);
            const F3 albedo = tex ? sample_point(tex, tw, th, p.x, p.z) : albedoConst;
            F3 Lr = mk(0.f, 0.f, 0.f);
            if (!occluded(nodes, tris, root, p, n, L, mk(0.f, 0.f, 0.f))) {
                float contrib = lightIntensity / d2 * std::fmax(dot(normalize(toL), n), 0.0f);
                contrib = std::fmin(contrib, radianceClamp);
                F3 xyz = mk(cmf_x(lambda) / kIntegralCmfY, cmf_y(lambda) / kIntegralCmfY, cmf_z(lambda) / kIntegralCmfY);
                F3 srgb = xyz2srgblinear(xyz);
                Lr = Lr + (albedo / kPi) * srgb * contrib / p_lambda;
            }
            st3(fd, p);
            st3(fd + 3, n);
            st3(fd + 6, albedo);
            fd[9] = lambda;
            acc[0] += Lr.x;
            acc[1] += Lr.y;
            acc[2] += Lr.z;
            acc[3] += 1.0f;
        }
    }
}

// ---------------------------------------------------------------- solver primitives
// dtype: 0 = float, 1 = double.  params: 2K values of that dtype (in/out).
int pzo_solve_constraints(int K, int dtype, void* params, const double* p_beg, const double* p_end,
                          const Triangle* tris, const TriangleAttrib* attribs, double eta, uint32_t events,
                          int maxIter, double tol, int warmup, int* itersOut)
{
#define PZO_SOLVE(KK)                                                                                              \
    case KK:                                                                                                       \
        if (dtype == 0)                                                                                            \
            return solve_constraints<float, KK>((float*)params, mk((float)p_beg[0], (float)p_beg[1], (float)p_beg[2]), \
                                                mk((float)p_end[0], (float)p_end[1], (float)p_end[2]), tris, attribs, \
                                                (float)eta, events, maxIter, (float)tol, warmup, itersOut);        \
        return solve_constraints<double, KK>((double*)params, mk(p_beg[0], p_beg[1], p_beg[2]),                   \
                                             mk(p_end[0], p_end[1], p_end[2]), tris, attribs, eta, events, maxIter, \
                                             tol, warmup, itersOut);
    switch (K) {
        PZO_SOLVE(1)
        PZO_SOLVE(2)
        PZO_SOLVE(3)
        PZO_SOLVE(4)
        default: return -1;
    }
#undef PZO_SOLVE
}

double pzo_contributable_throughput(int K, int dtype, const void* params, const double* p_beg, const double* p_end,
                                    const Triangle* tris, const TriangleAttrib* attribs, uint32_t events,
                                    const InternalNode* nodes, const Triangle* sceneTris, uint32_t root, double eta)
{
#define PZO_THR(KK)                                                                                              \
    case KK:                                                                                                     \
        if (dtype == 0)                                                                                          \
            return contributable_throughput<float, KK>((const float*)params,                                     \
                                                       mk((float)p_beg[0], (float)p_beg[1], (float)p_beg[2]),    \
                                                       mk((float)p_end[0], (float)p_end[1], (float)p_end[2]),    \
                                                       tris, attribs, events, nodes, sceneTris, root, (float)eta); \
        return contributable_throughput<double, KK>((const double*)params, mk(p_beg[0], p_beg[1], p_beg[2]),   \
                                                    mk(p_end[0], p_end[1], p_end[2]), tris, attribs, events,   \
                                                    nodes, sceneTris, root, eta);
    switch (K) {
        PZO_THR(1)
        PZO_THR(2)
        PZO_THR(3)
        PZO_THR(4)
        default: return -1.0;
    }
#undef PZO_THR
}

double pzo_dAdw(int dtype, const double* ro, const double* rd, const double* p_end, const Triangle* tris,
                const TriangleAttrib* attribs, uint32_t events, double eta)
{
    if (dtype == 0)
        return dAdw<float>(mk((float)ro[0], (float)ro[1], (float)ro[2]), mk((float)rd[0], (float)rd[1], (float)rd[2]),
                           mk((float)p_end[0], (float)p_end[1], (float)p_end[2]), tris, attribs, events, (float)eta);
    return dAdw<double>(mk(ro[0], ro[1], ro[2]), mk(rd[0], rd[1], rd[2]), mk(p_end[0], p_end[1], p_end[2]), tris,
                        attribs, events, eta);
}

// ---------------------------------------------------------------- binned specular render
// For every (pixel, slot) pair and every wavelength bin: solve from the photon's
// barycentrics (solveSpecularPath<K>, main_gpu.cu:418-486, with lambda fixed to the
// bin centre), validate, weigh by dAdw, clamp and accumulate into
// spectral[pixel * nBins + bin].  Stats: [0] solves, [1] converged, [2] contributing.
// dtype 0 = float, 1 = double (the FP64 reference image).
}  // extern "C"
template <class T, int K>
static void render_pairs(const int32_t* pairs, int64_t nPairs, const int32_t* slotTris, const float* slotParams,
                         const float* firstDiffuse, const InternalNode* nodes, uint32_t root, const Triangle* tris,
                         const TriangleAttrib* attribs, F3 L, float lightIntensity, float radianceClamp,
                         uint32_t events, const float* etas, int nBins, int maxIter, float tol, int warmup,
                         float* spectral, int64_t* stats)
{
    std::atomic<int64_t> conv{0}, contrib{0};
    int nt = omp_get_max_threads();
    std::vector<std::vector<float>> partial(nt);
#pragma omp parallel
    {
        int64_t lc = 0, lk = 0;
#pragma omp for schedule(dynamic, 64)
        for (int64_t q = 0; q < nPairs; q++) {
            int px = pairs[2 * q], slot = pairs[2 * q + 1];
            const float* fd = firstDiffuse + 10 * (size_t)px;
            V3<T> p = mk((T)fd[0], (T)fd[1], (T)fd[2]);
            V3<T> n = mk((T)fd[3], (T)fd[4], (T)fd[5]);
            Triangle tk[K];
            TriangleAttrib ak[K];
            for (int k = 0; k < K; k++) { tk[k] = tris[slotTris[4 * slot + k]]; ak[k] = attribs[slotTris[4 * slot + k]]; }
            for (int b = 0; b < nBins; b++) {
                T prm[2 * K];
                for (int i = 0; i < 2 * K; i++) prm[i] = (T)slotParams[8 * slot + i];
                T eta = (T)etas[b];
                V3<T> Lt = mk((T)L.x, (T)L.y, (T)L.z);
                bool ok = solve_constraints<T, K>(prm, Lt, p, tk, ak, eta, events, maxIter, (T)tol, warmup);
                if (!ok) continue;
                lc++;
                T thr = contributable_throughput<T, K>(prm, Lt, p, tk, ak, events, nodes, tris, root, eta);
                if (!(T(0) < thr)) continue;
                lk++;
                T dadw = dAdw<T>(Lt, get_vertex<T>(0, tk, prm) - Lt, p, tk, ak, events, eta);
                T cosv = std::fmax(dot(normalize(get_vertex<T>(K - 1, tk, prm) - p), n), T(0));
                T c = thr * (T)lightIntensity / dadw * cosv;
                c = std::fmin(c, (T)radianceClamp);
#pragma omp atomic
                spectral[(size_t)px * nBins + b] += (float)c;
            }
        }
        conv += lc;
        contrib += lk;
    }
    stats[0] = nPairs * nBins;
    stats[1] = conv;
    stats[2] = contrib;
}
// The reference's own solve mode (solveSpecularPath<K>, main_gpu.cu:418-483): one thread per
// (pixel, tuple) with the pixel's sampled wavelength from the eye pass (FirstDiffuse.lambda),
// eta = cauchy(lambda), and the clamped contribution weighted into linear sRGB by the CMFs
// and the wavelength pdf, added to the pixel's float4 accumulator (RGB; w untouched).
template <class T, int K>
static void render_pairs_rgb(const int32_t* pairs, int64_t nPairs, const int32_t* slotTris, const float* slotParams,
                             const float* firstDiffuse, const InternalNode* nodes, uint32_t root, const Triangle* tris,
                             const TriangleAttrib* attribs, F3 L, float lightIntensity, float radianceClamp,
                             uint32_t events, float cauchyA, float cauchyB, int maxIter, float tol, int warmup,
                             float* accum, int64_t* stats)
{
    int64_t conv = 0, contrib = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : conv, contrib)
    for (int64_t q = 0; q < nPairs; q++) {
        int px = pairs[2 * q], slot = pairs[2 * q + 1];
        const float* fd = firstDiffuse + 10 * (size_t)px;
        V3<T> p = mk((T)fd[0], (T)fd[1], (T)fd[2]);
        V3<T> n = mk((T)fd[3], (T)fd[4], (T)fd[5]);
        const F3 R = mk(fd[6], fd[7], fd[8]);
        const float lambda = fd[9];
        Triangle tk[K];
        TriangleAttrib ak[K];
        for (int k = 0; k < K; k++) { tk[k] = tris[slotTris[4 * slot + k]]; ak[k] = attribs[slotTris[4 * slot + k]]; }
        T prm[2 * K];
        for (int i = 0; i < 2 * K; i++) prm[i] = (T)slotParams[8 * slot + i];
        const float p_lambda = cmf_y_pdf(lambda);
        const T eta = (T)cauchy(cauchyA, cauchyB, lambda);
        V3<T> Lt = mk((T)L.x, (T)L.y, (T)L.z);
        if (!solve_constraints<T, K>(prm, Lt, p, tk, ak, eta, events, maxIter, (T)tol, warmup)) continue;
        conv++;
        T thr = contributable_throughput<T, K>(prm, Lt, p, tk, ak, events, nodes, tris, root, eta);
        if (!(T(0) < thr)) continue;
        contrib++;
        T dadw = dAdw<T>(Lt, get_vertex<T>(0, tk, prm) - Lt, p, tk, ak, events, eta);
        T cosv = std::fmax(dot(normalize(get_vertex<T>(K - 1, tk, prm) - p), n), T(0));
        T c = thr * (T)lightIntensity / dadw * cosv;
        c = std::fmin(c, (T)radianceClamp);
        const float cf = (float)c;
        const F3 xyz = mk(cmf_x(lambda) / kIntegralCmfY, cmf_y(lambda) / kIntegralCmfY, cmf_z(lambda) / kIntegralCmfY);
        const F3 Lr = (R / kPi) * xyz2srgblinear(xyz) * cf / p_lambda;
        float* a = accum + 4 * (size_t)px;
#pragma omp atomic
        a[0] += Lr.x;
#pragma omp atomic
        a[1] += Lr.y;
#pragma omp atomic
        a[2] += Lr.z;
    }
    stats[0] = nPairs;
    stats[1] = conv;
    stats[2] = contrib;
}
// Per-path contributions (before the clamp; 0 = rejected) of every (pair, bin), for the
// finite-difference references of the adjoint: the set of accepted paths can then be held
// fixed across the perturbed renders.
template <class T, int K>
static void render_each(const int32_t* pairs, int64_t nPairs, const int32_t* slotTris, const float* slotParams,
                        const float* firstDiffuse, const InternalNode* nodes, uint32_t root, const Triangle* tris,
                        const TriangleAttrib* attribs, F3 L, float lightIntensity, uint32_t events, const float* etas,
                        int nBins, int maxIter, float tol, int warmup, double* out)
{
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t q = 0; q < nPairs; q++) {
        int px = pairs[2 * q], slot = pairs[2 * q + 1];
        const float* fd = firstDiffuse + 10 * (size_t)px;
        V3<T> p = mk((T)fd[0], (T)fd[1], (T)fd[2]);
        V3<T> n = mk((T)fd[3], (T)fd[4], (T)fd[5]);
        Triangle tk[K];
        TriangleAttrib ak[K];
        for (int k = 0; k < K; k++) { tk[k] = tris[slotTris[4 * slot + k]]; ak[k] = attribs[slotTris[4 * slot + k]]; }
        for (int b = 0; b < nBins; b++) {
            double c = 0.0;
            T prm[2 * K];
            for (int i = 0; i < 2 * K; i++) prm[i] = (T)slotParams[8 * slot + i];
            T eta = (T)etas[b];
            V3<T> Lt = mk((T)L.x, (T)L.y, (T)L.z);
            if (solve_constraints<T, K>(prm, Lt, p, tk, ak, eta, events, maxIter, (T)tol, warmup)) {
                T thr = contributable_throughput<T, K>(prm, Lt, p, tk, ak, events, nodes, tris, root, eta);
                if (T(0) < thr) {
                    T dadw = dAdw<T>(Lt, get_vertex<T>(0, tk, prm) - Lt, p, tk, ak, events, eta);
                    T cosv = std::fmax(dot(normalize(get_vertex<T>(K - 1, tk, prm) - p), n), T(0));
                    c = (double)(thr * (T)lightIntensity / dadw * cosv);
                }
            }
            out[(size_t)q * nBins + b] = c;
        }
    }
}

extern "C" {

int pzo_render_pairs(int K, int dtype, const int32_t* pairs, int64_t nPairs, const int32_t* slotTris,
                     const float* slotParams, const float* firstDiffuse, const InternalNode* nodes, uint32_t root,
                     const Triangle* tris, const TriangleAttrib* attribs, const float* p_light, float lightIntensity,
                     float radianceClamp, uint32_t events, const float* etas, int nBins, int maxIter, float tol,
                     int warmup, float* spectral, int64_t* stats)
{
    F3 L = ld3(p_light);
#define PZO_R(KK)                                                                                                   \
    case KK:                                                                                                        \
        if (dtype == 0)                                                                                             \
            render_pairs<float, KK>(pairs, nPairs, slotTris, slotParams, firstDiffuse, nodes, root, tris, attribs, L, \
                                    lightIntensity, radianceClamp, events, etas, nBins, maxIter, tol, warmup,       \
                                    spectral, stats);                                                               \
        else                                                                                                        \
            render_pairs<double, KK>(pairs, nPairs, slotTris, slotParams, firstDiffuse, nodes, root, tris, attribs, \
                                     L, lightIntensity, radianceClamp, events, etas, nBins, maxIter, tol, warmup,   \
                                     spectral, stats);                                                              \
        return 0;
    switch (K) {
        PZO_R(1)
        PZO_R(2)
        PZO_R(3)
        PZO_R(4)
        default: return -1;
    }
#undef PZO_R
}

int pzo_render_pairs_rgb(int K, int dtype, const int32_t* pairs, int64_t nPairs, const int32_t* slotTris,
                         const float* slotParams, const float* firstDiffuse, const InternalNode* nodes, uint32_t root,
                         const Triangle* tris, const TriangleAttrib* attribs, const float* p_light,
                         float lightIntensity, float radianceClamp, uint32_t events, float cauchyA, float cauchyB,
                         int maxIter, float tol, int warmup, float* accum, int64_t* stats)
{
    F3 L = ld3(p_light);
#define PZO_RGB(KK)                                                                                                  \
    case KK:                                                                                                         \
        if (dtype == 0)                                                                                              \
            render_pairs_rgb<float, KK>(pairs, nPairs, slotTris, slotParams, firstDiffuse, nodes, root, tris,        \
                                        attribs, L, lightIntensity, radianceClamp, events, cauchyA, cauchyB,        \
                                        maxIter, tol, warmup, accum, stats);                                        \
        else                                                                                                         \
            render_pairs_rgb<double, KK>(pairs, nPairs, slotTris, slotParams, firstDiffuse, nodes, root, tris,       \
                                         attribs, L, lightIntensity, radianceClamp, events, cauchyA, cauchyB,       \
                                         maxIter, tol, warmup, accum, stats);                                       \
        return 0;
    switch (K) {
        PZO_RGB(1)
        PZO_RGB(2)
        PZO_RGB(3)
        PZO_RGB(4)
        default: return -1;
    }
#undef PZO_RGB
}

// CIE 2015 10-degree CMFs and the wavelength sampling (pk.h:960-1012): 0 x, 1 y, 2 z,
// 3 pdf of the CMF-y logistic, 4 its inverse CDF.
float pzo_cmf(int which, float nm)
{
    switch (which) {
        case 0: return cmf_x(nm);
        case 1: return cmf_y(nm);
        case 2: return cmf_z(nm);
        case 3: return cmf_y_pdf(nm);
        case 4: return cmf_y_sample(nm);
    }
    return 0.0f;
}

// pack (main_gpu.cu:499-513): accumulator / count -> sRGB OETF -> RGBA8.
void pzo_pack(const float* accum, int n, uint32_t* pixels)
{
    for (int i = 0; i < n; i++) {
        const float* a = accum + 4 * (size_t)i;
        pixels[i] = pack_rgba(srgb_oetf(a[0] / a[3]), srgb_oetf(a[1] / a[3]), srgb_oetf(a[2] / a[3]), 1.0f);
    }
}

// Binned spectral image -> linear sRGB and RGBA8: (albedo / pi) * sum_b S_b * srgb(lambda_b)
// * dlambda, lambda_b the bin centres (the quadrature of the reference's Monte Carlo estimate
// (R / pi) srgb(lambda) contrib / p(lambda), main_gpu.cu:473-478).  No reference counterpart.
void pzo_resolve_spectral(const float* spectral, int n, int nBins, float lambdaMin, float lambdaMax,
                          const float* albedo3, float* rgb4, uint32_t* pixels)
{
    const float w = (lambdaMax - lambdaMin) / (float)nBins;
    const F3 albedo = ld3(albedo3);
    for (int i = 0; i < n; i++) {
        F3 c = mk(0.f, 0.f, 0.f);
        for (int b = 0; b < nBins; b++) {
            const float lam = lambdaMin + ((float)b + 0.5f) * w;
            const F3 xyz = mk(cmf_x(lam) / kIntegralCmfY, cmf_y(lam) / kIntegralCmfY, cmf_z(lam) / kIntegralCmfY);
            c = c + xyz2srgblinear(xyz) * (spectral[(size_t)i * nBins + b] * w);
        }
        c = (albedo / kPi) * c;
        if (rgb4) {
            rgb4[4 * (size_t)i + 0] = c.x;
            rgb4[4 * (size_t)i + 1] = c.y;
            rgb4[4 * (size_t)i + 2] = c.z;
            rgb4[4 * (size_t)i + 3] = 1.0f;
        }
        if (pixels) pixels[i] = pack_rgba(srgb_oetf(c.x), srgb_oetf(c.y), srgb_oetf(c.z), 1.0f);
    }
}

int pzo_render_each(int K, int dtype, const int32_t* pairs, int64_t nPairs, const int32_t* slotTris,
                    const float* slotParams, const float* firstDiffuse, const InternalNode* nodes, uint32_t root,
                    const Triangle* tris, const TriangleAttrib* attribs, const float* p_light, float lightIntensity,
                    uint32_t events, const float* etas, int nBins, int maxIter, float tol, int warmup, double* out)
{
    F3 L = ld3(p_light);
#define PZO_E(KK)                                                                                                  \
    case KK:                                                                                                       \
        if (dtype == 0)                                                                                            \
            render_each<float, KK>(pairs, nPairs, slotTris, slotParams, firstDiffuse, nodes, root, tris, attribs, L, \
                                   lightIntensity, events, etas, nBins, maxIter, tol, warmup, out);                \
        else                                                                                                       \
            render_each<double, KK>(pairs, nPairs, slotTris, slotParams, firstDiffuse, nodes, root, tris, attribs,  \
                                    L, lightIntensity, events, etas, nBins, maxIter, tol, warmup, out);            \
        return 0;
    switch (K) {
        PZO_E(1)
        PZO_E(2)
        PZO_E(3)
        PZO_E(4)
        default: return -1;
    }
#undef PZO_E
}

// ---------------------------------------------------------------- interval + path cuts
void pzo_interval_square(const float* lu, float* out) { Intr r = isquare(Intr{lu[0], lu[1]}); out[0] = r.l; out[1] = r.u; }
void pzo_interval_normalize(const float* box6, float* out6)
{
    Intr3 r = inormalize(Intr3{{box6[0], box6[1]}, {box6[2], box6[3]}, {box6[4], box6[5]}});
    out6[0] = r.x.l; out6[1] = r.x.u; out6[2] = r.y.l; out6[3] = r.y.u; out6[4] = r.z.l; out6[5] = r.z.u;
}
float pzo_fresnel(const float* wi, const float* n, float eta) { return fresnel_exact_norm_free(ld3(wi), ld3(n), eta); }
int pzo_refract(const float* wi, const float* n, float eta, float* wo)
{
    F3 r;
    bool ok = refraction_norm_free(&r, ld3(wi), ld3(n), eta);
    if (ok) st3(wo, r);
    return ok ? 1 : 0;
}

// Normal bounds (main.cpp:250-295): out 13 floats per internal node
// {normalBounds[0] (6), normalBounds[1] (6), counter}.
void pzo_normal_bounds(const InternalNode* internals, int nInternals, const Triangle* tris,
                       const TriangleAttrib* attribs, InternalNormalBound* out)
{
    std::vector<InternalNormalBound> nb;
    build_normal_bounds(nb, internals, nInternals, tris, attribs);
    std::memcpy(out, nb.data(), sizeof(InternalNormalBound) * (size_t)nInternals);
}

// traverseAdmissibleNodes<K> (pk.h:1760-2220).  Writes K indices per admissible tuple
// in callback order.  Returns count (negative on overflow); visited = node tuples popped.
int64_t pzo_path_cuts(int K, uint32_t events, float eta, const float* p_beg, const float* p_end,
                      const InternalNode* internals, const InternalNormalBound* nbs, const Triangle* tris,
                      const TriangleAttrib* attribs, uint32_t root, int32_t* out, int64_t cap, uint64_t* visited)
{
    int64_t n = 0;
    auto cb = [&](const int* idx) {
        if (n < cap)
            for (int k = 0; k < K; k++) out[n * K + k] = idx[k];
        n++;
    };
    F3 a = ld3(p_beg), b = ld3(p_end);
    switch (K) {
        case 1: traverse_admissible_nodes<1>(events, eta, a, b, internals, nbs, tris, attribs, root, cb, visited); break;
        case 2: traverse_admissible_nodes<2>(events, eta, a, b, internals, nbs, tris, attribs, root, cb, visited); break;
        case 3: traverse_admissible_nodes<3>(events, eta, a, b, internals, nbs, tris, attribs, root, cb, visited); break;
        case 4: traverse_admissible_nodes<4>(events, eta, a, b, internals, nbs, tris, attribs, root, cb, visited); break;
        default: return 0;
    }
    return n > cap ? -n : n;
}

// Subdivision solve (pz_oracle_subdiv.hpp): roots of every tuple row {q, tri[0..K)},
// sorted by (tuple, bin, depth, path).  The rows index tris / attribs; visibility runs
// through nodes over scene_tris.  stats[8]: boxes tested, culled, leaves, (leaf, bin)
// pairs excluded, solves, converged, outside their box, roots.  Returns the root count
// (negative on overflow).
int64_t pzo_subdivide_solve(int K, uint32_t events, const float* p_beg, const float* p_end, const uint32_t* tuples,
                            uint32_t n_tuples, const float* etas, int n_bins, int max_depth, float eps,
                            int max_iterations, float cost_tolerance, int warm_up, const Triangle* tris,
                            const TriangleAttrib* attribs, const InternalNode* nodes, const Triangle* scene_tris,
                            uint32_t root, void* out, int64_t cap, uint64_t* stats)
{
    subdiv::Params P{max_depth, eps, max_iterations, cost_tolerance, warm_up};
    const F3 a = ld3(p_beg);
    const F3* ends = reinterpret_cast<const F3*>(p_end);
    std::vector<std::vector<subdiv::Root>> rows(n_tuples);
    std::vector<std::array<uint64_t, 8>> st(n_tuples);
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t r = 0; r < (int64_t)n_tuples; r++) {
        st[r].fill(0);
        const uint32_t ri = (uint32_t)r;
        switch (K) {
            case 1: subdiv::solve_row<1>(ri, tuples, events, a, ends, etas, n_bins, P, tris, attribs, nodes, scene_tris, root, rows[r], st[r].data()); break;
            case 2: subdiv::solve_row<2>(ri, tuples, events, a, ends, etas, n_bins, P, tris, attribs, nodes, scene_tris, root, rows[r], st[r].data()); break;
            case 3: subdiv::solve_row<3>(ri, tuples, events, a, ends, etas, n_bins, P, tris, attribs, nodes, scene_tris, root, rows[r], st[r].data()); break;
            case 4: subdiv::solve_row<4>(ri, tuples, events, a, ends, etas, n_bins, P, tris, attribs, nodes, scene_tris, root, rows[r], st[r].data()); break;
            default: break;
        }
    }
    int64_t n = 0;
    subdiv::Root* o = static_cast<subdiv::Root*>(out);
    for (int j = 0; j < 8; j++) stats[j] = 0;
    for (uint32_t r = 0; r < n_tuples; r++) {
        for (int j = 0; j < 8; j++) stats[j] += st[r][j];
        auto& v = rows[r];
        std::sort(v.begin(), v.end(), [](const subdiv::Root& x, const subdiv::Root& y) {
            return std::make_tuple(x.bin, x.depth, x.path) < std::make_tuple(y.bin, y.depth, y.path);
        });
        for (const auto& x : v) {
            if (n < cap) o[n] = x;
            n++;
        }
    }
    return n > cap ? -n : n;
}

// Contributions of subdivision roots to a binned spectral image (the tail of
// solveSpecularPath<K>, main_gpu.cu:466-486, at each root's bin): rows' query = pixel of
// first_diffuse (10 floats per pixel).  Accumulates in root order.
void pzo_subdivide_contribute(int K, uint32_t events, const float* p_beg, float light_intensity, float radiance_clamp,
                              const uint32_t* tuples, const void* roots, int64_t n_roots, const float* first_diffuse,
                              const float* etas, int n_bins, const Triangle* tris, const TriangleAttrib* attribs,
                              float* spectral)
{
    const subdiv::Root* rs = static_cast<const subdiv::Root*>(roots);
    const F3 L = ld3(p_beg);
    for (int64_t i = 0; i < n_roots; i++) {
        const subdiv::Root& r = rs[i];
        const uint32_t* t = tuples + (size_t)r.tuple * (1 + K);
        const uint32_t px = t[0];
        Triangle tk[4];
        TriangleAttrib ak[4];
        for (int k = 0; k < K; k++) { tk[k] = tris[t[1 + k]]; ak[k] = attribs[t[1 + k]]; }
        const float* fd = first_diffuse + 10 * (size_t)px;
        const F3 p = mk(fd[0], fd[1], fd[2]), n = mk(fd[3], fd[4], fd[5]);
        const float eta = etas[r.bin];
        const float dadw = dAdw<float>(L, get_vertex<float>(0, tk, r.params) - L, p, tk, ak, events, eta);
        const float cosv = std::fmax(dot(normalize(get_vertex<float>(K - 1, tk, r.params) - p), n), 0.0f);
        float c = r.throughput * light_intensity / dadw * cosv;
        c = std::fmin(c, radiance_clamp);
        spectral[(size_t)px * n_bins + r.bin] += c;
    }
}

// One directed-rounding operation of the subdivision oracle (op 0 add, 1 sub, 2 mul,
// 3 div (downward only), 4 sqrt; up = 1 rounds toward +inf, 0 toward -inf).
float pzo_directed(int op, int up, float a, float b)
{
    switch (op) {
        case 0: return up ? subdiv::add_u(a, b) : subdiv::add_d(a, b);
        case 1: return up ? subdiv::sub_u(a, b) : subdiv::sub_d(a, b);
        case 2: return up ? subdiv::mul_u(a, b) : subdiv::mul_d(a, b);
        case 3: return subdiv::div_d(a, b);
        default: return up ? subdiv::sqrt_u(a) : subdiv::sqrt_d(a);
    }
}

}  // extern "C"
