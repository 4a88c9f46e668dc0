// ref_harness.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Thin C entry points over the reference's OWN CPU code (minimum_lbvh.h, pk.h,
// interval.h, sen.h, saka.h, sobol.h, camera.h), compiled from the reference
// sources where they lie by oracle/build_ref.sh into oracle/_ref/libpzref.so.
// No reference source is copied into this repository: build_ref.sh generates
// pk_oracle.h from pk.h at build time by dropping the renderer class (which needs
// the absent graphics/Alembic libraries) and the GPU-builder define.
//
// The entry points mirror the pzo_* functions of oracle/pz_oracle_capi.cpp so the
// tests can pin the restatement against the reference.  Loops that in the
// reference live inside a kernel (photonTrace, main_gpu.cu:56-211) or inside the
// GL playground (normal bounds, main.cpp:250-295; CPU render loop,
// main.cpp:1584-1838) are written here around calls to the reference's functions.
#include <cmath>
#include <cstdio>
#include <stack>
#include <vector>

#include "interval.h"
#define ENABLE_PATH_CUTS
#include "pk_oracle.h"
#include "sobol.h"
#include "camera.h"

#include <omp.h>

bool g_bruteforce = false;  // pk.h:1758 declares it extern

using namespace minimum_lbvh;

static_assert(sizeof(Triangle) == 36, "layout");
static_assert(sizeof(TriangleAttrib) == 40, "layout");
static_assert(sizeof(InternalNode) == 64, "layout");

namespace {
inline float3 ld3(const float* p) { return make_float3(p[0], p[1], p[2]); }
inline void st3(float* p, float3 v) { p[0] = v.x; p[1] = v.y; p[2] = v.z; }
inline uint32_t nodeU32(NodeIndex n) { uint32_t u; memcpy(&u, &n, 4); return u; }
inline NodeIndex u32Node(uint32_t u) { NodeIndex n; memcpy(&n, &u, 4); return n; }
}  // namespace

extern "C" int pzr_version(void) { return 1; }
extern "C" void pzr_set_threads(int n) { if (n > 0) omp_set_num_threads(n); }
extern "C" int pzr_max_threads(void) { return omp_get_max_threads(); }

// GPU builder pipeline (minimum_lbvh.h:798-886, minimum_lbvh.cu) on the host, using the
// reference's AABB, Morton, delta and build_lbvh functions and a stable sort (the
// order the GPU onesweep sort produces).
extern "C" int pzr_build_bvh(const Triangle* tris, int n, uint32_t opt, InternalNode* nodes_out, uint32_t* root_out,
                  uint64_t* sorted_out, uint8_t* deltas_out, float* aabb_out6)
{
    AABB scene;
    scene.setEmpty();
    for (int i = 0; i < n; i++)
        for (int j = 0; j < 3; j++) scene.extend(tris[i].vs[j]);
    std::vector<IndexedMorton> m(n);
    for (int i = 0; i < n; i++) {
        Triangle tri = tris[i];
        float3 center = (tri.vs[0] + tri.vs[1] + tri.vs[2]) / 3.0f;
        if (opt & BUILD_OPTION_USE_NORMAL) {  // GPU packing, minimum_lbvh.cu:79-86
            float3 ng = normalOf(tri);
            AABB unit = {{-1, -1, -1}, {+1, +1, +1}};
            uint32_t nMorton = (uint32_t)(unit.encodeMortonCode(ng) >> 31);
            uint32_t pMorton = (uint32_t)(scene.encodeMortonCode(center) >> 31);
            m[i].morton = (nMorton & 0xFFFFFFC0) | (pMorton >> 26);
        } else {
            m[i].morton = (uint32_t)(scene.encodeMortonCode(center) >> 31);
        }
        m[i].index = i;
    }
    std::stable_sort(m.begin(), m.end(), [](IndexedMorton a, IndexedMorton b) { return a.morton < b.morton; });
    std::vector<uint8_t> deltas(n > 1 ? n - 1 : 0);
    for (int i = 0; i + 1 < n; i++) deltas[i] = (uint8_t)delta(m[i].morton, m[i + 1].morton);
    std::vector<InternalNode> internals(n > 1 ? n - 1 : 1);
    memset(internals.data(), 0xFF, sizeof(InternalNode) * internals.size());
    NodeIndex root = NodeIndex::invalid();
    if (n > 1)
        for (int i = 0; i < n; i++) build_lbvh(&root, internals.data(), tris, n, deltas.data(), i, m[i].index);
    if (n == 1) root = NodeIndex(m[0].index, true);
    if (n > 1) memcpy(nodes_out, internals.data(), sizeof(InternalNode) * (n - 1));
    *root_out = nodeU32(root);
    if (sorted_out)
        for (int i = 0; i < n; i++) sorted_out[i] = (uint64_t)m[i].morton | ((uint64_t)m[i].index << 32);
    if (deltas_out && n > 1) memcpy(deltas_out, deltas.data(), n - 1);
    if (aabb_out6) { st3(aabb_out6, scene.lower); st3(aabb_out6 + 3, scene.upper); }
    return 0;
}

// BVHCPUBuilder::build as the reference ships it (unstable std::sort, CPU key packing
// for USE_NORMAL).  Used as the CPU baseline and, for inputs without duplicate keys, as a
// cross-check of the pipeline above.
extern "C" int pzr_cpu_builder(const Triangle* tris, int n, uint32_t opt, InternalNode* nodes_out, uint32_t* root_out)
{
    BVHCPUBuilder b;
    b.build(tris, n, opt);
    memcpy(nodes_out, b.m_internals.data(), sizeof(InternalNode) * b.m_internals.size());
    *root_out = nodeU32(b.m_rootNode);
    return b.m_internals.size() == (size_t)(n - 1) ? 0 : -1;
}

extern "C" void pzr_trace_closest(const InternalNode* nodes, uint32_t root, const Triangle* tris, int n, const float* ro,
                       const float* rd, float* t, float* uv, uint32_t* tri, float* ng)
{
#pragma omp parallel
    {
        std::vector<NodeIndex> stack(256);
#pragma omp for schedule(dynamic, 256)
        for (int i = 0; i < n; i++) {
            Hit h;
            float3 o = ld3(ro + 3 * i), d = ld3(rd + 3 * i);
            intersect_stackfull(&h, nodes, tris, u32Node(root), o, d, invRd(d), stack.data());
            t[i] = h.t;
            uv[2 * i] = h.uv.x;
            uv[2 * i + 1] = h.uv.y;
            tri[i] = h.triangleIndex;
            st3(ng + 3 * i, h.ng);
        }
    }
}

extern "C" void pzr_trace_any(const InternalNode* nodes, uint32_t root, const Triangle* tris, int n, const float* ro,
                   const float* rd, const float* tmax, uint8_t* hit_out)
{
#pragma omp parallel for schedule(dynamic, 256)
    for (int i = 0; i < n; i++) {
        Hit h;
        h.t = tmax[i];
        float3 o = ld3(ro + 3 * i), d = ld3(rd + 3 * i);
        intersect_escape_link(&h, nodes, tris, u32Node(root), o, d, invRd(d), RAY_QUERY_ANY);
        hit_out[i] = h.t < tmax[i] ? 1 : 0;
    }
}

// One photon per (triangle, j): the body of photonTrace (main_gpu.cu:56-211) around
// the reference's functions.  Record layout as pzo_photon_trace.
struct PhotonRecordC { uint32_t ev; int32_t tris[4]; float params[8]; float p[3]; };

extern "C" int64_t pzr_photon_trace(const InternalNode* nodes, uint32_t rootU, const Triangle* triangles,
                         const TriangleAttrib* attribs, int nTris, const float* p_light_, float eta_min, float eta_max,
                         int iteration, float minThroughput, int photonsPerTri, PhotonRecordC* out, int64_t capacity)
{
    float3 p_light = ld3(p_light_);
    NodeIndex rootNode = u32Node(rootU);
    std::vector<std::vector<PhotonRecordC>> perTri(nTris);
#pragma omp parallel
    {
        std::vector<NodeIndex> stack(256);
#pragma omp for schedule(dynamic, 16)
        for (int iTri = 0; iTri < nTris; iTri++) {
            if (attribs[iTri].material == Material::Diffuse) continue;
            Triangle tri = triangles[iTri];
            float3 ng = unnormalizedNormalOf(tri);
            float3 ns = attribs[iTri].shadingNormals[0];
            ng *= dot(ng, ns);
            if (dot(ng, p_light - tri.vs[0]) < 0.0f) continue;
            enum { K = PHOTON_TRACE_MAX_DEPTH };
            for (int j = 0; j < photonsPerTri; j++) {
                float2 params = {};
                sobol::shuffled_scrambled_sobol_2d(&params.x, &params.y, j, iteration, iTri, 789);
                params = square2triangle(params);
                float2 eta_random;
                sobol::shuffled_scrambled_sobol_2d(&eta_random.x, &eta_random.y, j, iteration, iTri, 178);
                float eta = lerp(eta_min, eta_max, eta_random.x);
                float3 e0 = tri.vs[1] - tri.vs[0];
                float3 e1 = tri.vs[2] - tri.vs[0];
                float3 p = tri.vs[0] + e0 * params.x + e1 * params.y;
                float3 ro = p_light;
                float3 rd = p - p_light;
                EventDescriptor eDescriptor;
                bool admissiblePath = false;
                int triIndices[K] = {};
                float parameters[K * 2] = {};
                float3 p_final = {};
                float throughtput = 1.0f;
                for (int d = 0; d < K + 1; d++) {
                    Hit hit;
                    intersect_stackfull(&hit, nodes, triangles, rootNode, ro, rd, invRd(rd), stack.data());
                    if (hit.t == MINIMUM_LBVH_FLT_MAX) break;
                    TriangleAttrib attrib = attribs[hit.triangleIndex];
                    Material m = attrib.material;
                    float3 p_hit = ro + rd * hit.t;
                    float3 ns2 = attrib.shadingNormals[0] + (attrib.shadingNormals[1] - attrib.shadingNormals[0]) * hit.uv.x +
                                 (attrib.shadingNormals[2] - attrib.shadingNormals[0]) * hit.uv.y;
                    if (m == Material::Diffuse) {
                        if (d == 0) break;
                        admissiblePath = true;
                        p_final = p_hit;
                        break;
                    }
                    if (d == K) break;
                    float3 wi = -rd;
                    triIndices[d] = hit.triangleIndex;
                    parameters[d * 2] = hit.uv.x;
                    parameters[d * 2 + 1] = hit.uv.y;
                    float2 random;
                    sobol::shuffled_scrambled_sobol_2d(&random.x, &random.y, j, d, iTri, iteration);
                    float reflectance = fresnel_exact_norm_free(wi, ns2, eta);
                    Event e = Event::R;
                    if (m == Material::Mirror) e = Event::R;
                    else if (m == Material::Dielectric) e = random.x < reflectance ? Event::R : Event::T;
                    eDescriptor.push_back(e);
                    float sign = 1.0f;
                    float3 wo;
                    if (e == Event::R) {
                        wo = reflection(wi, ns2);
                        if (m == Material::Dielectric) throughtput *= reflectance;
                    } else {
                        if (refraction_norm_free(&wo, wi, ns2, eta) == false) break;
                        sign = -1.0f;
                        throughtput *= 1.0f - reflectance;
                    }
                    if (0.0f < dot(hit.ng, wi) * dot(hit.ng, wo) * sign) {
                        float3 offset_dir = normalize(hit.ng * dot(hit.ng, wo));
                        ro = p_hit + offset_dir * rayOffsetScale(p_hit);
                        rd = wo;
                        continue;
                    }
                    break;
                }
                if (admissiblePath && minThroughput < throughtput) {
                    PhotonRecordC c;
                    c.ev = eDescriptor.asU32();
                    memcpy(c.tris, triIndices, sizeof(c.tris));
                    memcpy(c.params, parameters, sizeof(c.params));
                    st3(c.p, p_final);
                    perTri[iTri].push_back(c);
                }
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

// The reference's host PathCache (pk.h:227-402): records inserted in order.
extern "C" int64_t pzr_cache_build(const PhotonRecordC* recs, int64_t n, uint32_t capacity, float step, uint32_t* hashOfPath,
                        uint32_t* cellHash, uint32_t* events, int32_t* trisOut, float* paramsOut)
{
    if (capacity != PathCache::CACHE_STORAGE_COUNT) return -1;  // the reference's capacity is fixed
    PathCache c(TYPED_BUFFER_HOST);
    c.init(step);
    for (int64_t i = 0; i < n; i++) {
        EventDescriptor e;
        e.m_events = recs[i].ev & 0xFFFFFF;
        e.m_size = recs[i].ev >> 24;
        int t[4];
        memcpy(t, recs[i].tris, sizeof(t));
        float prm[8];
        memcpy(prm, recs[i].params, sizeof(prm));
        c.store(ld3(recs[i].p), t, prm, e);
    }
    for (uint32_t i = 0; i < capacity; i++) {
        hashOfPath[i] = c.m_hashsOfPath[i];
        if (hashOfPath[i] == 0) {
            cellHash[i] = 0; events[i] = 0;
            for (int d = 0; d < 4; d++) trisOut[4 * i + d] = 0;
            for (int d = 0; d < 8; d++) paramsOut[8 * i + d] = 0.0f;
            continue;
        }
        const auto& p = c.m_pathes[i];
        cellHash[i] = p.hashOfP;
        events[i] = p.eDescriptor.asU32();
        int K = p.eDescriptor.size();
        for (int d = 0; d < 4; d++) trisOut[4 * i + d] = d < K ? p.tris[d] : 0;
        for (int d = 0; d < 8; d++) paramsOut[8 * i + d] = d < 2 * K ? p.parameters[d] : 0.0f;
    }
    return (int64_t)c.m_numberOfCached[0];
}

extern "C" uint32_t pzr_spacial_hash(const float* p, float step) { return spacial_hash(ld3(p), step); }

extern "C" void pzr_lookat(const float* eye, const float* center, const float* up, float fovy, int w, int h, float* out9)
{
    RayGenerator g;
    g.lookat(ld3(eye), ld3(center), ld3(up), fovy, w, h);
    st3(out9, g.m_origin);
    st3(out9 + 3, g.m_right);
    st3(out9 + 6, g.m_up);
}
extern "C" void pzr_shoot(const float* gen9, float u, float v, float* ro, float* rd)
{
    RayGenerator g;
    g.m_origin = ld3(gen9);
    g.m_right = ld3(gen9 + 3);
    g.m_up = ld3(gen9 + 6);
    float3 o, d;
    g.shoot(&o, &d, u, v);
    st3(ro, o);
    st3(rd, d);
}

extern "C" void pzr_sobol(uint32_t index, uint32_t p0, uint32_t p1, uint32_t p2, float* xy)
{
    sobol::shuffled_scrambled_sobol_2d(&xy[0], &xy[1], index, p0, p1, p2);
}

template <int K>
static int solveK(float* params, const float* pb, const float* pe, Triangle* tris, TriangleAttrib* attribs, float eta,
                  uint32_t ev, int maxIter, float tol, int warmup, int* iters)
{
    EventDescriptor e;
    e.m_events = ev & 0xFFFFFF;
    e.m_size = ev >> 24;
    int last = -1;
    bool conv = false;
    auto cb = [&](int iter, bool c) { last = iter; conv = c; };
    bool r = solveConstraints<K>(params, ld3(pb), ld3(pe), tris, attribs, eta, e, maxIter, tol, warmup, cb);
    if (iters) *iters = last;
    (void)conv;
    return r ? 1 : 0;
}
extern "C" int pzr_solve_constraints(int K, float* params, const float* pb, const float* pe, Triangle* tris, TriangleAttrib* attribs,
                          float eta, uint32_t ev, int maxIter, float tol, int warmup, int* iters)
{
    switch (K) {
        case 1: return solveK<1>(params, pb, pe, tris, attribs, eta, ev, maxIter, tol, warmup, iters);
        case 2: return solveK<2>(params, pb, pe, tris, attribs, eta, ev, maxIter, tol, warmup, iters);
        case 3: return solveK<3>(params, pb, pe, tris, attribs, eta, ev, maxIter, tol, warmup, iters);
        case 4: return solveK<4>(params, pb, pe, tris, attribs, eta, ev, maxIter, tol, warmup, iters);
    }
    return -1;
}

extern "C" float pzr_contributable_throughput(int K, float* params, const float* pb, const float* pe, Triangle* tris,
                                   TriangleAttrib* attribs, uint32_t ev, const InternalNode* nodes,
                                   const Triangle* sceneTris, uint32_t root, float eta)
{
    EventDescriptor e;
    e.m_events = ev & 0xFFFFFF;
    e.m_size = ev >> 24;
    switch (K) {
        case 1: return contributableThroughput<1>(params, ld3(pb), ld3(pe), tris, attribs, e, nodes, sceneTris, u32Node(root), eta);
        case 2: return contributableThroughput<2>(params, ld3(pb), ld3(pe), tris, attribs, e, nodes, sceneTris, u32Node(root), eta);
        case 3: return contributableThroughput<3>(params, ld3(pb), ld3(pe), tris, attribs, e, nodes, sceneTris, u32Node(root), eta);
        case 4: return contributableThroughput<4>(params, ld3(pb), ld3(pe), tris, attribs, e, nodes, sceneTris, u32Node(root), eta);
    }
    return -1.0f;
}

extern "C" float pzr_dAdw(const float* ro, const float* rd, const float* pe, Triangle* tris, TriangleAttrib* attribs, uint32_t ev, float eta)
{
    EventDescriptor e;
    e.m_events = ev & 0xFFFFFF;
    e.m_size = ev >> 24;
    return dAdw(ld3(ro), ld3(rd), ld3(pe), tris, attribs, e, eta);
}

extern "C" float pzr_fresnel(const float* wi, const float* n, float eta) { return fresnel_exact_norm_free(ld3(wi), ld3(n), eta); }
extern "C" int pzr_refract(const float* wi, const float* n, float eta, float* wo)
{
    float3 r;
    bool ok = refraction_norm_free(&r, ld3(wi), ld3(n), eta);
    if (ok) st3(wo, r);
    return ok ? 1 : 0;
}
extern "C" void pzr_interval_square(const float* lu, float* out)
{
    interval::intr r = interval::square(interval::intr(lu[0], lu[1]));
    out[0] = r.l;
    out[1] = r.u;
}
extern "C" void pzr_interval_normalize(const float* b, float* out)
{
    interval::intr3 r = interval::normalize(interval::make_intr3({b[0], b[1]}, {b[2], b[3]}, {b[4], b[5]}));
    out[0] = r.x.l; out[1] = r.x.u; out[2] = r.y.l; out[3] = r.y.u; out[4] = r.z.l; out[5] = r.z.u;
}
extern "C" float pzr_cmf(int which, float nm)
{
    switch (which) {
        case 0: return CIE_2015_10deg::cmf_x(nm);
        case 1: return CIE_2015_10deg::cmf_y(nm);
        case 2: return CIE_2015_10deg::cmf_z(nm);
        case 3: return CIE_2015_10deg::cmf_y_pdf(nm);
        case 4: return CIE_2015_10deg::cmf_y_sample(nm);
    }
    return 0.0f;
}

// Normal bounds: the loop of main.cpp:250-295 over the reference's types.
extern "C" void pzr_normal_bounds(const InternalNode* internals, int nInternals, const Triangle* tris, const TriangleAttrib* attribs,
                       InternalNormalBound* out)
{
    std::vector<InternalNormalBound> nb(nInternals);
    memset(nb.data(), 0, sizeof(InternalNormalBound) * nInternals);
    for (uint32_t i = 0; i < (uint32_t)nInternals; i++) {
        for (int j = 0; j < 2; j++) {
            NodeIndex me = internals[i].children[j];
            if (!me.m_isLeaf) continue;
            NodeIndex parent(i, false);
            AABB normalBound;
            normalBound.setEmpty();
            const TriangleAttrib& attrib = attribs[me.m_index];
            for (int k = 0; k < 3; k++) normalBound.extend(attrib.shadingNormals[k]);
            while (parent != NodeIndex::invalid()) {
                int childIndex = internals[parent.m_index].children[0] == me ? 0 : 1;
                nb[parent.m_index].normalBounds[childIndex] = normalBound;
                uint32_t vindex = nb[parent.m_index].counter++;
                if (vindex == 0) break;
                normalBound.extend(nb[parent.m_index].normalBounds[childIndex ^ 0x1]);
                me = parent;
                parent = internals[me.m_index].parent;
            }
        }
    }
    memcpy(out, nb.data(), sizeof(InternalNormalBound) * nInternals);
}

template <int K>
static int64_t pathCutsK(uint32_t ev, float eta, const float* pb, const float* pe, InternalNode* internals,
                         InternalNormalBound* nbs, Triangle* tris, TriangleAttrib* attribs, uint32_t root, int32_t* out,
                         int64_t cap)
{
    EventDescriptor e;
    e.m_events = ev & 0xFFFFFF;
    e.m_size = ev >> 24;
    int64_t n = 0;
    traverseAdmissibleNodes<K>(e, eta, ld3(pb), ld3(pe), internals, nbs, tris, attribs, u32Node(root),
                               [&](AdmissibleTriangles<K> a) {
                                   if (n < cap)
                                       for (int k = 0; k < K; k++) out[n * K + k] = a.indices[k];
                                   n++;
                               });
    return n > cap ? -n : n;
}
extern "C" int64_t pzr_path_cuts(int K, uint32_t ev, float eta, const float* pb, const float* pe, InternalNode* internals,
                      InternalNormalBound* nbs, Triangle* tris, TriangleAttrib* attribs, uint32_t root, int32_t* out,
                      int64_t cap)
{
    switch (K) {
        case 1: return pathCutsK<1>(ev, eta, pb, pe, internals, nbs, tris, attribs, root, out, cap);
        case 2: return pathCutsK<2>(ev, eta, pb, pe, internals, nbs, tris, attribs, root, out, cap);
        case 3: return pathCutsK<3>(ev, eta, pb, pe, internals, nbs, tris, attribs, root, out, cap);
        case 4: return pathCutsK<4>(ev, eta, pb, pe, internals, nbs, tris, attribs, root, out, cap);
    }
    return 0;
}

// CPU caustic render over a (pixel, slot) work list, per wavelength bin: the
// per-path sequence of main.cpp:1813-1825 / main_gpu.cu:456-483 with the
// reference's solveConstraints / contributableThroughput / dAdw.
template <int K>
static void renderK(const int32_t* pairs, int64_t nPairs, const int32_t* slotTris, const float* slotParams,
                    const float* fdv, const InternalNode* nodes, uint32_t rootU, const Triangle* tris,
                    const TriangleAttrib* attribs, float3 L, float I, float clampV, uint32_t ev, const float* etas,
                    int nBins, int maxIter, float tol, int warmup, float* spectral, int64_t* stats)
{
    EventDescriptor e;
    e.m_events = ev & 0xFFFFFF;
    e.m_size = ev >> 24;
    NodeIndex root = u32Node(rootU);
    int64_t conv = 0, contrib = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : conv, contrib)
    for (int64_t q = 0; q < nPairs; q++) {
        int px = pairs[2 * q], slot = pairs[2 * q + 1];
        const float* fd = fdv + 10 * (size_t)px;
        float3 p = ld3(fd), n = ld3(fd + 3);
        Triangle tk[K];
        TriangleAttrib ak[K];
        for (int k = 0; k < K; k++) { tk[k] = tris[slotTris[4 * slot + k]]; ak[k] = attribs[slotTris[4 * slot + k]]; }
        for (int b = 0; b < nBins; b++) {
            float prm[2 * K];
            for (int i = 0; i < 2 * K; i++) prm[i] = slotParams[8 * slot + i];
            float eta = etas[b];
            if (!solveConstraints<K>(prm, L, p, tk, ak, eta, e, maxIter, tol, warmup)) continue;
            conv++;
            float thr = contributableThroughput<K>(prm, L, p, tk, ak, e, nodes, tris, root, eta);
            if (!(0.0f < thr)) continue;
            contrib++;
            float dadw = dAdw(L, getVertex(0, tk, prm) - L, p, tk, ak, e, eta);
            float c = thr * I / dadw * fmaxf(dot(normalize(getVertex(K - 1, tk, prm) - p), n), 0.0f);
            c = fminf(c, clampV);
#pragma omp atomic
            spectral[(size_t)px * nBins + b] += c;
        }
    }
    stats[0] = nPairs * nBins;
    stats[1] = conv;
    stats[2] = contrib;
}
extern "C" int pzr_render_pairs(int K, const int32_t* pairs, int64_t nPairs, const int32_t* slotTris, const float* slotParams,
                     const float* fd, const InternalNode* nodes, uint32_t root, const Triangle* tris,
                     const TriangleAttrib* attribs, const float* p_light, float I, float clampV, uint32_t ev,
                     const float* etas, int nBins, int maxIter, float tol, int warmup, float* spectral, int64_t* stats)
{
    float3 L = ld3(p_light);
    switch (K) {
        case 1: renderK<1>(pairs, nPairs, slotTris, slotParams, fd, nodes, root, tris, attribs, L, I, clampV, ev, etas, nBins, maxIter, tol, warmup, spectral, stats); return 0;
        case 2: renderK<2>(pairs, nPairs, slotTris, slotParams, fd, nodes, root, tris, attribs, L, I, clampV, ev, etas, nBins, maxIter, tol, warmup, spectral, stats); return 0;
        case 3: renderK<3>(pairs, nPairs, slotTris, slotParams, fd, nodes, root, tris, attribs, L, I, clampV, ev, etas, nBins, maxIter, tol, warmup, spectral, stats); return 0;
        case 4: renderK<4>(pairs, nPairs, slotTris, slotParams, fd, nodes, root, tris, attribs, L, I, clampV, ev, etas, nBins, maxIter, tol, warmup, spectral, stats); return 0;
    }
    return -1;
}


// The reference's own solve mode on the CPU: solveSpecularPath<K> (main_gpu.cu:418-483)
// written as a loop over the work list around the reference's functions -- eta from the
// pixel's sampled wavelength (CauchyDispersion), solveConstraints, contributableThroughput,
// dAdw, the CMF weights (CIE_2015_10deg, xyz2srgblinear) and the wavelength pdf -- adding
// RGB into a float4 accumulator per pixel (w untouched).
template <int K>
static void renderRgbK(const int32_t* pairs, int64_t nPairs, const int32_t* slotTris, const float* slotParams,
                       const float* fdv, const InternalNode* nodes, uint32_t rootU, const Triangle* tris,
                       const TriangleAttrib* attribs, float3 L, float I, float clampV, uint32_t ev,
                       CauchyDispersion cauchy, int maxIter, float tol, int warmup, float* accum, int64_t* stats)
{
    EventDescriptor e;
    e.m_events = ev & 0xFFFFFF;
    e.m_size = ev >> 24;
    NodeIndex root = u32Node(rootU);
    int64_t conv = 0, contrib = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : conv, contrib)
    for (int64_t q = 0; q < nPairs; q++) {
        int px = pairs[2 * q], slot = pairs[2 * q + 1];
        const float* fd = fdv + 10 * (size_t)px;
        float3 p = ld3(fd), n = ld3(fd + 3), R = ld3(fd + 6);
        float lambda = fd[9];
        Triangle tk[K];
        TriangleAttrib ak[K];
        for (int k = 0; k < K; k++) { tk[k] = tris[slotTris[4 * slot + k]]; ak[k] = attribs[slotTris[4 * slot + k]]; }
        float prm[2 * K];
        for (int i = 0; i < 2 * K; i++) prm[i] = slotParams[8 * slot + i];
        float p_lambda = CIE_2015_10deg::cmf_y_pdf(lambda);
        float eta = cauchy(lambda);
        if (!solveConstraints<K>(prm, L, p, tk, ak, eta, e, maxIter, tol, warmup)) continue;
        conv++;
        float thr = contributableThroughput<K>(prm, L, p, tk, ak, e, nodes, tris, root, eta);
        if (!(0.0f < thr)) continue;
        contrib++;
        float dadw = dAdw(L, getVertex(0, tk, prm) - L, p, tk, ak, e, eta);
        float c = thr * I / dadw * fmaxf(dot(normalize(getVertex(K - 1, tk, prm) - p), n), 0.0f);
        c = fminf(c, clampV);
        float3 xyz = {CIE_2015_10deg::cmf_x(lambda) / INTEGRAL_OF_CMF_Y_IN_NM,
                      CIE_2015_10deg::cmf_y(lambda) / INTEGRAL_OF_CMF_Y_IN_NM,
                      CIE_2015_10deg::cmf_z(lambda) / INTEGRAL_OF_CMF_Y_IN_NM};
        float3 srgblinear = xyz2srgblinear(xyz);
        float3 Lr = (R / PI) * srgblinear * c / p_lambda;
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
extern "C" int pzr_render_pairs_rgb(int K, const int32_t* pairs, int64_t nPairs, const int32_t* slotTris,
                                    const float* slotParams, const float* fd, const InternalNode* nodes, uint32_t root,
                                    const Triangle* tris, const TriangleAttrib* attribs, const float* p_light, float I,
                                    float clampV, uint32_t ev, float cauchyA, float cauchyB, int maxIter, float tol,
                                    int warmup, float* accum, int64_t* stats)
{
    float3 L = ld3(p_light);
    CauchyDispersion c(cauchyA, cauchyB);
    switch (K) {
        case 1: renderRgbK<1>(pairs, nPairs, slotTris, slotParams, fd, nodes, root, tris, attribs, L, I, clampV, ev, c, maxIter, tol, warmup, accum, stats); return 0;
        case 2: renderRgbK<2>(pairs, nPairs, slotTris, slotParams, fd, nodes, root, tris, attribs, L, I, clampV, ev, c, maxIter, tol, warmup, accum, stats); return 0;
        case 3: renderRgbK<3>(pairs, nPairs, slotTris, slotParams, fd, nodes, root, tris, attribs, L, I, clampV, ev, c, maxIter, tol, warmup, accum, stats); return 0;
        case 4: renderRgbK<4>(pairs, nPairs, slotTris, slotParams, fd, nodes, root, tris, attribs, L, I, clampV, ev, c, maxIter, tol, warmup, accum, stats); return 0;
    }
    return -1;
}

// pack (main_gpu.cu:499-513) with the reference's srgb_oetf (pk.h:1023-1031); packRGBA
// (main_gpu.cu:9-14, device-only in the reference) is the 8-bit quantisation
// min(max(int(c * 255 + 0.5), 0), 255) per channel, truncating toward zero.
extern "C" void pzr_pack(const float* accum, int n, uint32_t* pixels)
{
    for (int i = 0; i < n; i++) {
        const float* a = accum + 4 * (size_t)i;
        int q[3];
        for (int c = 0; c < 3; c++) {
            const int v = (int)(srgb_oetf(a[c] / a[3]) * 255.0f + 0.5f);
            q[c] = v < 0 ? 0 : (v > 255 ? 255 : v);
        }
        pixels[i] = 0xFF000000u | ((uint32_t)q[2] << 16) | ((uint32_t)q[1] << 8) | (uint32_t)q[0];
    }
}
