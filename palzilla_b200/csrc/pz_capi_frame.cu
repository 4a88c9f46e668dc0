// pz_capi_frame.cu -- C ABI for ray queries, PathCache, photons, eye pass, work list,
// plain specular solve and resolve (include/palzilla_b200.h).
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "pz_batched_api.cuh"
#include "pz_cache.cuh"
#include "pz_capi_internal.h"
#include "pz_frame.cuh"
#include "pz_photon.cuh"
#include "pz_solve.cuh"
#include "pz_trace_api.cuh"

using namespace pz;

namespace {
inline cudaStream_t S(pz_stream_t s) { return reinterpret_cast<cudaStream_t>(s); }
inline float3 F3(pz_float3 v) { return make_float3(v.x, v.y, v.z); }
inline bool pow2(uint32_t x) { return x && !(x & (x - 1)); }
inline int done(cudaError_t e, const char* where)
{
    if (e != cudaSuccess) return cuda_fail(e, where);
    clear_error();
    return PZ_OK;
}
}  // namespace

extern "C" int pz_trace_closest(const pz_internal_node* internals_dev, const uint32_t* root_dev,
                                const pz_triangle* triangles_dev, int n_rays, const float* ro_dev, const float* rd_dev,
                                float* t_dev, float* uv_dev, uint32_t* tri_dev, float* ng_dev, uint32_t* status_dev,
                                pz_stream_t stream)
{
    if (n_rays < 0 || (n_rays > 0 && (!root_dev || !triangles_dev || !ro_dev || !rd_dev || !t_dev)))
        return fail(PZ_ERR_INVALID_ARGUMENT, "pz_trace_closest: bad argument");
    return done(launch_trace_closest(reinterpret_cast<const Node*>(internals_dev), root_dev,
                                     reinterpret_cast<const Tri*>(triangles_dev), (uint32_t)n_rays, ro_dev, rd_dev,
                                     t_dev, uv_dev, tri_dev, ng_dev, status_dev, S(stream)),
                "pz_trace_closest");
}

extern "C" int pz_trace_any(const pz_internal_node* internals_dev, const uint32_t* root_dev,
                            const pz_triangle* triangles_dev, int n_rays, const float* ro_dev, const float* rd_dev,
                            const float* tmax_dev, uint8_t* hit_dev, pz_stream_t stream)
{
    if (n_rays < 0 || (n_rays > 0 && (!root_dev || !triangles_dev || !ro_dev || !rd_dev || !tmax_dev || !hit_dev)))
        return fail(PZ_ERR_INVALID_ARGUMENT, "pz_trace_any: bad argument");
    return done(launch_trace_any(reinterpret_cast<const Node*>(internals_dev), root_dev,
                                 reinterpret_cast<const Tri*>(triangles_dev), (uint32_t)n_rays, ro_dev, rd_dev,
                                 tmax_dev, hit_dev, S(stream)),
                "pz_trace_any");
}

// ---------------------------------------------------------------- PathCache
extern "C" size_t pz_path_cache_bytes(uint32_t capacity) { return pow2(capacity) ? cache_bytes(capacity) : 0; }

// the store writes each slot's triangle indices and barycentrics as 16-byte vectors
static bool cache_ok(const void* cache_dev, uint32_t capacity)
{
    return cache_dev && (reinterpret_cast<uintptr_t>(cache_dev) & 15u) == 0 && pow2(capacity);
}

extern "C" int pz_path_cache_clear(void* cache_dev, uint32_t capacity, pz_stream_t stream)
{
    if (!cache_ok(cache_dev, capacity)) return fail(PZ_ERR_INVALID_ARGUMENT, "pz_path_cache_clear: bad argument");
    CacheView c = cache_view(cache_dev, capacity, 0.0f);
    cudaError_t e = cudaMemsetAsync(c.h, 0, sizeof(CacheHeader), S(stream));
    if (e == cudaSuccess) e = cudaMemsetAsync(c.hash, 0, sizeof(uint32_t) * (size_t)capacity, S(stream));
    return done(e, "pz_path_cache_clear");
}

extern "C" int pz_path_cache_views(void* cache_dev, uint32_t capacity, uint32_t** hash_dev, uint32_t** cell_dev,
                                   uint32_t** events_dev, int32_t** tris_dev, float** params_dev, uint32_t** count_dev)
{
    if (!cache_ok(cache_dev, capacity)) return fail(PZ_ERR_INVALID_ARGUMENT, "pz_path_cache_views: bad argument");
    CacheView c = cache_view(cache_dev, capacity, 0.0f);
    if (hash_dev) *hash_dev = c.hash;
    if (cell_dev) *cell_dev = c.cell;
    if (events_dev) *events_dev = c.event;
    if (tris_dev) *tris_dev = reinterpret_cast<int32_t*>(c.tris);
    if (params_dev) *params_dev = reinterpret_cast<float*>(c.params);
    if (count_dev) *count_dev = &c.h->count;
    clear_error();
    return PZ_OK;
}

// ---------------------------------------------------------------- photons
extern "C" int pz_photon_trace(const pz_internal_node* internals_dev, const uint32_t* root_dev,
                               const pz_triangle* triangles_dev, const pz_triangle_attrib* attribs_dev, int n_triangles,
                               int photons_per_triangle, pz_float3 p_light, float eta_min, float eta_max, int iteration,
                               float min_throughput, void* cache_dev, uint32_t cache_capacity, float cell_step,
                               pz_photon_record* records_dev, pz_stream_t stream)
{
    if (n_triangles < 0 || photons_per_triangle < 0 || !root_dev || (n_triangles > 0 && (!triangles_dev || !attribs_dev)))
        return fail(PZ_ERR_INVALID_ARGUMENT, "pz_photon_trace: bad argument");
    if (cache_dev && (!cache_ok(cache_dev, cache_capacity) || !(cell_step > 0.0f)))
        return fail(PZ_ERR_INVALID_ARGUMENT,
                    "pz_photon_trace: cache must be 16-byte aligned, capacity a power of two, step > 0");
    CacheView c{};
    if (cache_dev) c = cache_view(cache_dev, cache_capacity, cell_step);
    return done(launch_photons(reinterpret_cast<const Node*>(internals_dev), root_dev,
                               reinterpret_cast<const Tri*>(triangles_dev), reinterpret_cast<const Attrib*>(attribs_dev),
                               (uint32_t)n_triangles, (uint32_t)photons_per_triangle, F3(p_light), eta_min, eta_max,
                               iteration, min_throughput, c, reinterpret_cast<PhotonRecord*>(records_dev), S(stream)),
                "pz_photon_trace");
}

// ---------------------------------------------------------------- eye pass
extern "C" void pz_ray_generator_lookat(pz_ray_generator* g, pz_float3 eye, pz_float3 center, pz_float3 up, float fovy,
                                        int width, int height)
{
    // camera.h:10-22 on the host; 1/sqrt with correctly rounded operations as the
    // reference's host normalize, and the double-precision tan the reference calls.
    auto nrm = [](pz_float3 v) {
        float inv = 1.0f / std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z);
        return pz_float3{v.x * inv, v.y * inv, v.z * inv};
    };
    auto crs = [](pz_float3 a, pz_float3 b) {
        return pz_float3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
    };
    pz_float3 f = nrm(pz_float3{center.x - eye.x, center.y - eye.y, center.z - eye.z});
    pz_float3 s = nrm(crs(f, up));
    pz_float3 u = crs(s, f);
    float ty = (float)std::tan((double)(fovy * 0.5f));
    float tx = ty / (float)height * (float)width;
    g->origin = eye;
    g->right = pz_float3{s.x * tx, s.y * tx, s.z * tx};
    g->up = pz_float3{u.x * ty, u.y * ty, u.z * ty};
}

extern "C" int pz_solve_primary(float* accum_dev, pz_first_diffuse* first_diffuse_dev, int width, int height,
                                const pz_ray_generator* gen, const pz_lens_params* lens,
                                const pz_internal_node* internals_dev, const uint32_t* root_dev,
                                const pz_triangle* triangles_dev, const pz_triangle_attrib* attribs_dev,
                                pz_float3 p_light, float light_intensity, float radiance_clamp, float cauchy_a,
                                float cauchy_b, pz_float3 albedo, const pz_texture_rgbx* albedo_texture,
                                int iteration, uint32_t* status_dev, pz_stream_t stream)
{
    if (width < 0 || height < 0 || !gen || !accum_dev || !first_diffuse_dev || !root_dev || !triangles_dev ||
        !attribs_dev)
        return fail(PZ_ERR_INVALID_ARGUMENT, "pz_solve_primary: bad argument");
    Tex tex{nullptr, 0u, 0u};
    if (albedo_texture) {
        if (!albedo_texture->texels_dev || albedo_texture->width == 0 || albedo_texture->height == 0 ||
            (reinterpret_cast<uintptr_t>(albedo_texture->texels_dev) & 3))
            return fail(PZ_ERR_INVALID_ARGUMENT,
                        "pz_solve_primary: the albedo texture needs texels (4-byte aligned) and a non-zero size");
        tex = Tex{albedo_texture->texels_dev, albedo_texture->width, albedo_texture->height};
    }
    RayGen g{F3(gen->origin), F3(gen->right), F3(gen->up)};
    Lens l{0.6f, 0.05f, 0.0f};
    if (lens) l = Lens{lens->distance, lens->thickness, lens->R};
    return done(launch_primary(reinterpret_cast<float4*>(accum_dev), reinterpret_cast<FirstDiffuse*>(first_diffuse_dev),
                               width, height, g, l, reinterpret_cast<const Node*>(internals_dev), root_dev,
                               reinterpret_cast<const Tri*>(triangles_dev), reinterpret_cast<const Attrib*>(attribs_dev),
                               F3(p_light), light_intensity, radiance_clamp, cauchy_a, cauchy_b, F3(albedo), tex,
                               iteration, status_dev, S(stream)),
                "pz_solve_primary");
}

// ---------------------------------------------------------------- work list
extern "C" int pz_lookup_flatten(uint32_t events, pz_specular_path* paths_dev, uint64_t* indexed_dev,
                                 uint32_t* counter_dev, uint32_t capacity, const pz_first_diffuse* first_diffuse_dev,
                                 int n_pixels, void* cache_dev, uint32_t cache_capacity, float cell_step,
                                 pz_stream_t stream)
{
    if (n_pixels < 0 || !paths_dev || !indexed_dev || !counter_dev || !first_diffuse_dev ||
        !cache_ok(cache_dev, cache_capacity) || !(cell_step > 0.0f))
        return fail(PZ_ERR_INVALID_ARGUMENT, "pz_lookup_flatten: bad argument");
    return done(launch_lookup(events, reinterpret_cast<SpecularPath*>(paths_dev),
                              reinterpret_cast<unsigned long long*>(indexed_dev), counter_dev, capacity,
                              reinterpret_cast<const FirstDiffuse*>(first_diffuse_dev), n_pixels,
                              cache_view(cache_dev, cache_capacity, cell_step), S(stream)),
                "pz_lookup_flatten");
}

extern "C" int pz_reorder_specular_paths(const uint64_t* indexed_dev, pz_specular_path* dst_dev,
                                         const pz_specular_path* src_dev, uint32_t n, pz_stream_t stream)
{
    if (n > 0 && (!indexed_dev || !dst_dev || !src_dev))
        return fail(PZ_ERR_INVALID_ARGUMENT, "pz_reorder_specular_paths: bad argument");
    return done(launch_reorder(reinterpret_cast<const unsigned long long*>(indexed_dev),
                               reinterpret_cast<SpecularPath*>(dst_dev), reinterpret_cast<const SpecularPath*>(src_dev),
                               n, S(stream)),
                "pz_reorder_specular_paths");
}

// ---------------------------------------------------------------- solve
namespace pz {
int solve_args_from_desc(const pz_solve_desc* d, SolveArgs* a, const char* who)
{
    if (!d) return fail(PZ_ERR_INVALID_ARGUMENT, "%s: null descriptor", who);
    if (d->K < 1 || d->K > 4) return fail(PZ_ERR_INVALID_ARGUMENT, "%s: K must be 1..4 (got %d)", who, d->K);
    if ((int)(d->events >> 24) != d->K)
        return fail(PZ_ERR_INVALID_ARGUMENT, "%s: event descriptor size %u != K %d", who, d->events >> 24, d->K);
    if (!cache_ok(d->cache, d->cache_capacity) || !(d->cell_step > 0.0f))
        return fail(PZ_ERR_INVALID_ARGUMENT, "%s: bad cache", who);
    if (d->n_paths && (!d->paths || !d->first_diffuse || !d->root || !d->triangles || !d->attribs))
        return fail(PZ_ERR_INVALID_ARGUMENT, "%s: null buffer", who);
    if (d->spectral && (d->n_bins < 1 || !d->etas)) return fail(PZ_ERR_INVALID_ARGUMENT, "%s: bins need etas", who);
    if (!d->spectral && !d->accum) return fail(PZ_ERR_INVALID_ARGUMENT, "%s: need accum or spectral", who);
    a->accum = reinterpret_cast<float4*>(d->accum);
    a->spectral = d->spectral;
    a->etas = d->etas;
    a->nBins = d->spectral ? d->n_bins : 1;
    a->paths = reinterpret_cast<const SpecularPath*>(d->paths);
    a->nPaths = d->n_paths;
    a->fds = reinterpret_cast<const FirstDiffuse*>(d->first_diffuse);
    a->nodes = reinterpret_cast<const Node*>(d->internals);
    a->root = d->root;
    a->tris = reinterpret_cast<const Tri*>(d->triangles);
    a->attribs = reinterpret_cast<const Attrib*>(d->attribs);
    a->p_light = F3(d->p_light);
    a->lightIntensity = d->light_intensity;
    a->radianceClamp = d->radiance_clamp;
    a->cache = cache_view(d->cache, d->cache_capacity, d->cell_step);
    a->events = d->events;
    a->cauchyA = d->cauchy_a;
    a->cauchyB = d->cauchy_b;
    a->maxIterations = d->max_iterations > 0 ? d->max_iterations : 32;
    a->costTolerance = d->cost_tolerance > 0.0f ? d->cost_tolerance : 1.0e-10f;
    a->earlyTermWarmUp = d->early_term_warmup;
    a->stats = d->stats;
    a->roots = d->roots;
    return PZ_OK;
}
}  // namespace pz

extern "C" int pz_solve_specular_plain(const pz_solve_desc* desc, pz_stream_t stream)
{
    SolveArgs a;
    int r = solve_args_from_desc(desc, &a, "pz_solve_specular_plain");
    if (r != PZ_OK) return r;
    auto launch = desc->fma_contraction ? launch_solve_plain : launch_solve_plain_exact;
    return done(launch(desc->K, desc->spectral != nullptr, a, S(stream)), "pz_solve_specular_plain");
}

namespace {
// Scratch of one batched solve: 256-byte header | phase-1 records (one per work item) |
// plain-solve probes (three per work item) | phase-2 accepted roots | their blocks, each
// region 256-byte aligned.
struct BatchLayout {
    size_t records, probes, accepted, blocks, total;
};
inline size_t a256(size_t x) { return (x + 255) & ~(size_t)255; }
BatchLayout batch_layout(int K, uint64_t maxPaths, int nBins, size_t start)
{
    BatchLayout L;
    L.records = start;
    L.probes = L.records + a256((size_t)maxPaths * batched::record_bytes(K));
    L.accepted = L.probes + a256((size_t)maxPaths * 3 * batched::probe_bytes(K));
    L.blocks = L.accepted + a256((size_t)batched::accept_capacity(maxPaths, nBins) * batched::accepted_bytes(K));
    L.total = L.blocks + a256((size_t)batched::block_capacity(maxPaths) * batched::block_bytes());
    return L;
}
}  // namespace

extern "C" size_t pz_solve_batched_scratch_bytes(int K, uint64_t max_paths, int n_bins)
{
    if (K < 1 || K > 4 || n_bins < 1 || n_bins > 64) return 0;
    return batch_layout(K, max_paths, n_bins, 256).total;
}

extern "C" int pz_solve_specular_batched(const pz_solve_desc* desc, const uint32_t* n_paths_dev, void* scratch_dev,
                                         size_t scratch_bytes, int blocks_per_sm, pz_stream_t stream)
{
    batched::BatchArgs b;
    int r = solve_args_from_desc(desc, &b.s, "pz_solve_specular_batched");
    if (r != PZ_OK) return r;
    if (!desc->spectral || desc->n_bins < 1 || desc->n_bins > 64)
        return fail(PZ_ERR_INVALID_ARGUMENT, "pz_solve_specular_batched: binned mode with 1..64 bins required");
    const size_t need = pz_solve_batched_scratch_bytes(desc->K, desc->n_paths, desc->n_bins);
    if (!scratch_dev || scratch_bytes < need)
        return fail(PZ_ERR_SCRATCH_TOO_SMALL, "pz_solve_specular_batched: scratch %zu < required %zu", scratch_bytes,
                    need);
    if (reinterpret_cast<uintptr_t>(scratch_dev) & 255)
        return fail(PZ_ERR_INVALID_ARGUMENT, "pz_solve_specular_batched: scratch needs 256-byte alignment");
    char* base = static_cast<char*>(scratch_dev);
    b.status = reinterpret_cast<uint32_t*>(base);
    b.workCounter = reinterpret_cast<unsigned long long*>(base + 8);
    b.recordCount = reinterpret_cast<unsigned long long*>(base + 16);
    b.workCounter2 = reinterpret_cast<unsigned long long*>(base + 24);
    b.recordCount2 = reinterpret_cast<unsigned long long*>(base + 32);
    const BatchLayout L = batch_layout(desc->K, desc->n_paths, desc->n_bins, 256);
    b.records = base + L.records;
    b.recordCapacity = desc->n_paths;
    b.probes = base + L.probes;
    b.accepted = base + L.accepted;
    b.acceptCapacity = batched::accept_capacity(desc->n_paths, desc->n_bins);
    b.blocks = base + L.blocks;
    b.blockCapacity = batched::block_capacity(desc->n_paths);
    b.p2 = reinterpret_cast<unsigned long long*>(base + 192);
    b.nPathsDev = n_paths_dev;
    static_assert(64 + 8 * batched::kNumCounters <= 192, "counters live in the scratch header before the phase-2 words");
    b.counters = reinterpret_cast<unsigned long long*>(base + 64);
    b.polishDet = desc->polish_det > 0.0f ? (double)desc->polish_det : 0.0;
    b.grazeCos = desc->graze_cos > 0.0f ? desc->graze_cos : 0.0f;
    b.continuation = desc->continuation;
    b.illDet = desc->fold_det < 0.0f ? 0.0f : (desc->fold_det == 0.0f ? batched::kDefaultFoldDet : desc->fold_det);
    if (desc->n_paths == 0) { clear_error(); return PZ_OK; }
    cudaError_t e = cudaMemsetAsync(base, 0, 256, S(stream));
    if (e == cudaSuccess) e = batched::launch_solve_batched(desc->K, b, blocks_per_sm > 0 ? blocks_per_sm : batched::kP2SolveBlocks,
                                                        S(stream));
    return done(e, "pz_solve_specular_batched");
}

// ---------------------------------------------------------------- resolve
extern "C" int pz_resolve(uint32_t* pixels_dev, const float* accum_dev, int n_pixels, pz_stream_t stream)
{
    if (n_pixels < 0 || (n_pixels > 0 && (!pixels_dev || !accum_dev)))
        return fail(PZ_ERR_INVALID_ARGUMENT, "pz_resolve: bad argument");
    return done(launch_pack(pixels_dev, reinterpret_cast<const float4*>(accum_dev), n_pixels, S(stream)), "pz_resolve");
}

extern "C" int pz_resolve_spectral(float* rgb_dev, uint32_t* pixels_dev, const float* spectral_dev, int n_pixels,
                                   int n_bins, float lambda_min, float lambda_max, pz_float3 albedo, pz_stream_t stream)
{
    if (n_pixels < 0 || n_bins < 1 || (n_pixels > 0 && !spectral_dev))
        return fail(PZ_ERR_INVALID_ARGUMENT, "pz_resolve_spectral: bad argument");
    return done(launch_resolve_spectral(reinterpret_cast<float4*>(rgb_dev), pixels_dev, spectral_dev, n_pixels, n_bins,
                                        lambda_min, lambda_max, F3(albedo), S(stream)),
                "pz_resolve_spectral");
}

// ---------------------------------------------------------------- batches of scenes
// Scratch: 256-byte header (status, work counter, record count, counters) | item offsets
// (n_scenes + 1) | scene table | phase-1 records | probes, each region 256-byte aligned.
namespace {
constexpr size_t kMultiHeader = 256;
inline size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }
struct MultiLayout {
    size_t offsets, table, records, probes, accepted, blocks, total;
};
MultiLayout multi_layout(int K, int nBins, uint32_t nScenes, uint64_t maxPaths)
{
    MultiLayout L;
    L.offsets = kMultiHeader;
    L.table = L.offsets + align256(8 * ((size_t)nScenes + 1));
    const BatchLayout B = batch_layout(K, maxPaths, nBins, L.table + align256(sizeof(batched::SceneArgs) * (size_t)nScenes));
    L.records = B.records;
    L.probes = B.probes;
    L.accepted = B.accepted;
    L.blocks = B.blocks;
    L.total = B.total;
    return L;
}

// tunings found by pz_solve_multi_autotune, by (K, bins, log2 of the item capacity)
std::mutex g_tune_mutex;
std::map<std::tuple<int, int, int>, pz_batch_tuning> g_tunings;
std::tuple<int, int, int> tune_key(int K, int nBins, uint64_t maxPaths)
{
    int lg = 0;
    while ((1ull << lg) < maxPaths && lg < 63) lg++;
    return std::make_tuple(K, nBins, lg);
}
}  // namespace

extern "C" size_t pz_solve_multi_scratch_bytes(int K, int n_bins, uint32_t n_scenes, uint64_t max_paths_total)
{
    if (K < 1 || K > 4 || n_bins < 1 || n_bins > 64 || n_scenes == 0) return 0;
    return multi_layout(K, n_bins, n_scenes, max_paths_total).total;
}

extern "C" int pz_solve_multi_prepare(const pz_solve_desc* descs, const uint32_t* const* n_paths_dev, uint32_t n_scenes,
                                      void* scratch_dev, size_t scratch_bytes, pz_stream_t stream)
{
    if (!descs || n_scenes == 0) return fail(PZ_ERR_INVALID_ARGUMENT, "pz_solve_multi_prepare: no scenes");
    const int K = descs[0].K, nb = descs[0].n_bins;
    uint64_t total = 0;
    std::vector<batched::SceneArgs> table(n_scenes);
    for (uint32_t i = 0; i < n_scenes; i++) {
        const pz_solve_desc& d = descs[i];
        if (d.K != K || d.n_bins != nb || !d.spectral || nb < 1 || nb > 64)
            return fail(PZ_ERR_INVALID_ARGUMENT,
                        "pz_solve_multi_prepare: scene %u: every scene needs the same K and 1..64 bins, binned mode", i);
        int r = solve_args_from_desc(&d, &table[i].s, "pz_solve_multi_prepare");
        if (r != PZ_OK) return r;
        table[i].s.stats = nullptr;
        table[i].nPathsDev = n_paths_dev ? n_paths_dev[i] : nullptr;
        total += d.n_paths;
    }
    const MultiLayout L = multi_layout(K, nb, n_scenes, total);
    if (!scratch_dev || scratch_bytes < L.total)
        return fail(PZ_ERR_SCRATCH_TOO_SMALL, "pz_solve_multi_prepare: scratch %zu < required %zu", scratch_bytes, L.total);
    if (reinterpret_cast<uintptr_t>(scratch_dev) & 255)
        return fail(PZ_ERR_INVALID_ARGUMENT, "pz_solve_multi_prepare: scratch needs 256-byte alignment");
    char* base = static_cast<char*>(scratch_dev);
    cudaError_t e = cudaMemcpyAsync(base + L.table, table.data(), sizeof(batched::SceneArgs) * n_scenes,
                                    cudaMemcpyHostToDevice, S(stream));
    if (e == cudaSuccess) e = cudaStreamSynchronize(S(stream));
    return done(e, "pz_solve_multi_prepare");
}

static int multi_args(int K, int n_bins, uint32_t n_scenes, uint64_t total, void* scratch_dev, size_t scratch_bytes,
                      unsigned long long* stats_dev, batched::BatchArgs* b, unsigned long long** offsets,
                      const char* who)
{
    if (K < 1 || K > 4 || n_bins < 1 || n_bins > 64 || n_scenes == 0)
        return fail(PZ_ERR_INVALID_ARGUMENT, "%s: bad K / bins / scene count", who);
    const MultiLayout L = multi_layout(K, n_bins, n_scenes, total);
    if (!scratch_dev || scratch_bytes < L.total)
        return fail(PZ_ERR_SCRATCH_TOO_SMALL, "%s: scratch %zu < required %zu", who, scratch_bytes, L.total);
    char* base = static_cast<char*>(scratch_dev);
    std::memset(&b->s, 0, sizeof(b->s));
    b->s.nBins = n_bins;
    b->s.stats = stats_dev;
    b->status = reinterpret_cast<uint32_t*>(base);
    b->workCounter = reinterpret_cast<unsigned long long*>(base + 8);
    b->recordCount = reinterpret_cast<unsigned long long*>(base + 16);
    b->workCounter2 = reinterpret_cast<unsigned long long*>(base + 24);
    b->recordCount2 = reinterpret_cast<unsigned long long*>(base + 32);
    b->counters = reinterpret_cast<unsigned long long*>(base + 64);
    b->records = base + L.records;
    b->recordCapacity = total;
    b->probes = base + L.probes;
    b->accepted = base + L.accepted;
    b->acceptCapacity = batched::accept_capacity(total, n_bins);
    b->blocks = base + L.blocks;
    b->blockCapacity = batched::block_capacity(total);
    b->p2 = reinterpret_cast<unsigned long long*>(base + 192);
    b->polishDet = 0.0;
    b->grazeCos = 0.0f;
    b->continuation = 0;
    b->illDet = batched::kDefaultFoldDet;
    b->scenes = reinterpret_cast<const batched::SceneArgs*>(base + L.table);
    b->nScenes = n_scenes;
    *offsets = reinterpret_cast<unsigned long long*>(base + L.offsets);
    b->offsets = *offsets;
    b->nPathsDev = nullptr;
    return PZ_OK;
}

static cudaError_t run_multi(int K, const batched::BatchArgs& b0, const pz_batch_tuning& t, unsigned long long* offsets,
                             void* scratch_dev, cudaStream_t s)
{
    batched::BatchArgs b = b0;
    b.chunk = t.p2_chunk;
    cudaError_t e = cudaMemsetAsync(scratch_dev, 0, kMultiHeader, s);
    if (e == cudaSuccess) e = batched::launch_solve_batched_multi(K, b, t.p1_blocks_per_sm, t.p2_blocks_per_sm, offsets, s);
    return e;
}

extern "C" int pz_solve_specular_multi(int K, int n_bins, uint32_t n_scenes, uint64_t max_paths_total,
                                       void* scratch_dev, size_t scratch_bytes, const pz_batch_tuning* tuning,
                                       unsigned long long* stats_dev, pz_stream_t stream)
{
    batched::BatchArgs b;
    unsigned long long* offsets = nullptr;
    int r = multi_args(K, n_bins, n_scenes, max_paths_total, scratch_dev, scratch_bytes, stats_dev, &b, &offsets,
                       "pz_solve_specular_multi");
    if (r != PZ_OK) return r;
    pz_batch_tuning t = {8, 2, batched::kP2ChunkDefault};
    if (tuning) {
        t = *tuning;
    } else {
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        auto it = g_tunings.find(tune_key(K, n_bins, max_paths_total));
        if (it != g_tunings.end()) t = it->second;
    }
    if (t.p1_blocks_per_sm < 1 || t.p1_blocks_per_sm > 32 || t.p2_blocks_per_sm < 1 || t.p2_blocks_per_sm > 2 ||
        t.p2_chunk < 1 || t.p2_chunk > batched::kP2ChunkMax)
        return fail(PZ_ERR_INVALID_ARGUMENT, "pz_solve_specular_multi: tuning out of range");
    return done(run_multi(K, b, t, offsets, scratch_dev, S(stream)), "pz_solve_specular_multi");
}

extern "C" int pz_solve_multi_autotune(int K, int n_bins, uint32_t n_scenes, uint64_t max_paths_total,
                                       void* scratch_dev, size_t scratch_bytes, unsigned long long* stats_dev,
                                       pz_batch_tuning* best_out, float* best_ms_out, pz_stream_t stream)
{
    batched::BatchArgs b;
    unsigned long long* offsets = nullptr;
    int r = multi_args(K, n_bins, n_scenes, max_paths_total, scratch_dev, scratch_bytes, stats_dev, &b, &offsets,
                       "pz_solve_multi_autotune");
    if (r != PZ_OK) return r;
    cudaStream_t s = S(stream);
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
        return fail(PZ_ERR_CUDA, "pz_solve_multi_autotune: events");
    pz_batch_tuning best = {8, 2, 1};
    float bestMs = 3.4e38f;
    cudaError_t e = run_multi(K, b, best, offsets, scratch_dev, s);  // warm-up
    const int p1s[] = {4, 8, 16}, p2s[] = {1, 2}, chunks[] = {1, 4};
    for (int p1 : p1s)
        for (int p2 : p2s)
            for (int c : chunks) {
                if (e != cudaSuccess) break;
                const pz_batch_tuning t = {p1, p2, c};
                e = cudaEventRecord(e0, s);
                if (e == cudaSuccess) e = run_multi(K, b, t, offsets, scratch_dev, s);
                if (e == cudaSuccess) e = cudaEventRecord(e1, s);
                if (e == cudaSuccess) e = cudaEventSynchronize(e1);
                float ms = 0.0f;
                if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
                if (e == cudaSuccess && ms < bestMs) {
                    bestMs = ms;
                    best = t;
                }
            }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e != cudaSuccess) return cuda_fail(e, "pz_solve_multi_autotune");
    {
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        g_tunings[tune_key(K, n_bins, max_paths_total)] = best;
    }
    if (best_out) *best_out = best;
    if (best_ms_out) *best_ms_out = bestMs;
    clear_error();
    return PZ_OK;
}
