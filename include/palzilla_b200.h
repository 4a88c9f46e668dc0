/*
 * palzilla_b200.h -- C ABI of the B200 (sm_100a) caustics hot path.
 *
 * Drop-in for the reference's LBVH / sort / photon / specular-solve path (Ushio/Palzilla).
 * Each entry point names the reference interface it replaces (file:line within the
 * reference project).  Conventions for every function:
 *   - returns PZ_OK (0) or a PZ_ERR_* code; pz_last_error() gives a message;
 *   - pointers named *_dev are device pointers owned by the caller; no function
 *     allocates or frees device memory unless its name says so (*_create / *_destroy);
 *   - work is enqueued on `stream` (a cudaStream_t; 0 = legacy default stream) and
 *     the call does not synchronise; device-side failures (overflow, a bounded wait
 *     that expired) are recorded in the status word at the start of the scratch
 *     buffer and read with pz_scratch_status();
 *   - scratch sizes come from the matching *_scratch_bytes() query; scratch need not
 *     be initialised.
 * Binary layouts of the structs below equal the reference's structs.
 */
#ifndef PALZILLA_B200_H
#define PALZILLA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define PZ_API __attribute__((visibility("default")))
#else
#define PZ_API
#endif

typedef struct CUstream_st* pz_stream_t; /* == cudaStream_t */

enum pz_status {
    PZ_OK = 0,
    PZ_ERR_INVALID_ARGUMENT = 1,
    PZ_ERR_SCRATCH_TOO_SMALL = 2,
    PZ_ERR_CUDA = 3,        /* a CUDA runtime call or launch failed */
    PZ_ERR_DEVICE = 4,      /* a kernel reported a failure in the status word */
    PZ_ERR_UNSUPPORTED = 5
};

/* status-word bits written by kernels */
#define PZ_DEVICE_ERR_SPIN_LIMIT 0x1u     /* a bounded spin wait expired (output undefined) */
#define PZ_DEVICE_ERR_CAPACITY 0x2u       /* a queue / table / list capacity was exceeded */
#define PZ_DEVICE_ERR_STACK 0x4u          /* a traversal stack would have overflowed */

/* minimum_lbvh::BUILD_OPTION, minimum_lbvh.h:42-46 */
#define PZ_BUILD_OPTION_USE_NORMAL 1u
#define PZ_BUILD_OPTION_CPU_PARALLEL 2u   /* accepted and ignored (CPU builder option) */

#define PZ_INVALID_NODE 0x7FFFFFFFu       /* NodeIndex::invalid(), minimum_lbvh.h:270-273 */

typedef struct pz_float3 { float x, y, z; } pz_float3;
/* minimum_lbvh::Triangle, minimum_lbvh.h:207-210 (36 B) */
typedef struct pz_triangle { pz_float3 vs[3]; } pz_triangle;
/* TriangleAttrib, pk.h:74-78 (40 B); material: 0 diffuse, 1 mirror, 2 dielectric (pk.h:67-72) */
typedef struct pz_triangle_attrib { int32_t material; pz_float3 shading_normals[3]; } pz_triangle_attrib;
/* minimum_lbvh::AABB, minimum_lbvh.h:220-261 */
typedef struct pz_aabb { pz_float3 lower, upper; } pz_aabb;
/* minimum_lbvh::InternalNode, minimum_lbvh.h:285-291 (64 B).  NodeIndex = u32 with the
 * index in bits 0..30 and the leaf flag in bit 31 (minimum_lbvh.h:263-274). */
typedef struct pz_internal_node {
    uint32_t children[2];
    pz_aabb aabbs[2];
    uint32_t parent;
    uint32_t context; /* escape link after the build */
} pz_internal_node;

/* ---------------------------------------------------------------- library */
PZ_API int pz_version(void);
/* Message for the last error returned on this thread ("" if none). */
PZ_API const char* pz_last_error(void);
/* Synchronises `stream`, then copies the status word at the start of `scratch_dev`
 * (any scratch buffer of this API) into *status_out. */
PZ_API int pz_scratch_status(const void* scratch_dev, uint32_t* status_out, pz_stream_t stream);

/* ---------------------------------------------------------------- onesweep radix sort
 * Replaces tinyhiponesweep::OnesweepSort::sort (tinyhiponesweep.h:592-668).
 * Stable LSD sort of n keys (key_bytes 4 or 8) on the 8-bit digits covering bits
 * [start_bit, start_bit + 8*ceil((end_bit-start_bit)/8)), carrying one u32 value per
 * key when values_dev != NULL.  The result ends in keys_dev / values_dev; tmp_keys_dev
 * (and tmp_values_dev) are ping-pong buffers of the same size. */
PZ_API size_t pz_onesweep_scratch_bytes(uint32_t n);
PZ_API int pz_onesweep_sort(void* keys_dev, uint32_t* values_dev, void* tmp_keys_dev, uint32_t* tmp_values_dev, uint32_t n,
                     int key_bytes, int start_bit, int end_bit, void* scratch_dev, size_t scratch_bytes,
                     pz_stream_t stream);

/* No reference counterpart (the reference's OnesweepSort owns and allocates its scratch).
 * The same sort as pz_onesweep_sort, with the scratch taken from a static device array of
 * this library instead of a caller buffer, for callers that cannot allocate device memory
 * at call time.  The array holds the 16 KiB header and the look-back rows for
 * PZ_ONESWEEP_STATIC_MAX_KEYS keys at the build's tile size: 1,695,744 bytes with the
 * default 5,120-key tiles, held in every CUDA context that loads the library until it
 * exits.  n > PZ_ONESWEEP_STATIC_MAX_KEYS is rejected with PZ_ERR_SCRATCH_TOO_SMALL before
 * any device work.  Every call looks up the array's address in the CUDA context current on
 * the calling thread (a __device__ array has one address per context), so hosts that make
 * their own contexts or re-create one after cudaDeviceReset are served too.  That look-up
 * allocates nothing, but the first call in a context may load the library's module into
 * it, so make that first call before any stream capture.  Nothing has to be zeroed by the
 * caller: each call clears what it uses on `stream`.  All calls in one context share the
 * array: calls whose GPU work can overlap (unordered streams) race; order them on one
 * stream.  When status_dev != NULL the sort's status word (PZ_DEVICE_ERR_* bits, 0 = ok)
 * is copied there on `stream` after the sort. */
#define PZ_ONESWEEP_STATIC_MAX_KEYS (1u << 22)
PZ_API int pz_onesweep_sort_static(void* keys_dev, uint32_t* values_dev, void* tmp_keys_dev, uint32_t* tmp_values_dev,
                            uint32_t n, int key_bytes, int start_bit, int end_bit, uint32_t* status_dev,
                            pz_stream_t stream);

/* ---------------------------------------------------------------- LBVH build
 * Replaces minimum_lbvh::BVHGPUBuilder::build (minimum_lbvh.h:798-886):
 * scene AABB, 32-bit Morton keys (upper 32 bits of a 63-bit code), stable radix
 * sort, deltas and the bottom-up (Apetrei) build with escape links.  Writes
 * n_triangles - 1 internal nodes and the root NodeIndex (device u32). */
PZ_API size_t pz_bvh_scratch_bytes(int n_triangles);
PZ_API int pz_bvh_build(const pz_triangle* triangles_dev, int n_triangles, uint32_t build_option,
                 pz_internal_node* internals_dev, uint32_t* root_dev, void* scratch_dev, size_t scratch_bytes,
                 pz_stream_t stream);
/* After pz_bvh_build on the same scratch: device pointers to the sorted
 * {morton (low 32 bits), triangle index (high 32)} u64 array (n entries), the u8
 * deltas (n - 1) and the scene AABB (decoded into *aabb_out on the host after a
 * stream synchronisation). */
PZ_API int pz_bvh_debug_views(void* scratch_dev, int n_triangles, const uint64_t** sorted_dev, const uint8_t** deltas_dev,
                       pz_aabb* aabb_out, pz_stream_t stream);


/* ---------------------------------------------------------------- ray queries
 * Batch closest-hit (intersect_stackfull, minimum_lbvh.h:927-988) and any-hit
 * (intersect_escape_link with RAY_QUERY_ANY, minimum_lbvh.h:1078-1152) queries.  Rays
 * are 3 floats per ray (origin, direction); hit outputs may be NULL except t_dev.  A
 * closest-hit miss reports t = FLT_MAX and triangle 0xFFFFFFFF; any-hit writes 1 when a
 * hit with t < tmax exists. */
PZ_API int pz_trace_closest(const pz_internal_node* internals_dev, const uint32_t* root_dev,
                            const pz_triangle* triangles_dev, int n_rays, const float* ro_dev, const float* rd_dev,
                            float* t_dev, float* uv_dev, uint32_t* tri_dev, float* ng_dev, uint32_t* status_dev,
                            pz_stream_t stream);
PZ_API int pz_trace_any(const pz_internal_node* internals_dev, const uint32_t* root_dev,
                        const pz_triangle* triangles_dev, int n_rays, const float* ro_dev, const float* rd_dev,
                        const float* tmax_dev, uint8_t* hit_dev, pz_stream_t stream);

/* ---------------------------------------------------------------- PathCache
 * Spatial hash of photon tuples (PathCache, pk.h:227-402) in one caller-owned buffer of
 * pz_path_cache_bytes(capacity) bytes starting on a 16-byte boundary; capacity must be a
 * power of two (the reference uses 2^22).  The status word (first 4 bytes) reports probe
 * overflow. */
PZ_API size_t pz_path_cache_bytes(uint32_t capacity);
/* PathCache::clear (pk.h:254-269): empties the table and the counters. */
PZ_API int pz_path_cache_clear(void* cache_dev, uint32_t capacity, pz_stream_t stream);
/* Device addresses of the cache arrays (hash, cell hash, event descriptor, 4 triangle
 * indices and 8 barycentrics per slot, stored-entry count). */
PZ_API int pz_path_cache_views(void* cache_dev, uint32_t capacity, uint32_t** hash_dev, uint32_t** cell_dev,
                               uint32_t** events_dev, int32_t** tris_dev, float** params_dev, uint32_t** count_dev);

/* ---------------------------------------------------------------- photon pass
 * photonTrace (main_gpu.cu:56-211): photons_per_triangle photons from every specular,
 * light-facing triangle (the reference's 256-thread block per triangle is 256), up to 4
 * Fresnel-sampled specular events to a diffuse landing, stored into the PathCache.
 * records_dev (n_triangles * photons_per_triangle records, or NULL) receives every
 * photon's path for inspection (ev = 0 when the photon produced none). */
typedef struct pz_photon_record { uint32_t ev; int32_t tris[4]; float params[8]; float p[3]; } pz_photon_record;
PZ_API int pz_photon_trace(const pz_internal_node* internals_dev, const uint32_t* root_dev,
                           const pz_triangle* triangles_dev, const pz_triangle_attrib* attribs_dev, int n_triangles,
                           int photons_per_triangle, pz_float3 p_light, float eta_min, float eta_max, int iteration,
                           float min_throughput, void* cache_dev, uint32_t cache_capacity, float cell_step,
                           pz_photon_record* records_dev, pz_stream_t stream);

/* ---------------------------------------------------------------- eye pass */
typedef struct pz_ray_generator { pz_float3 origin, right, up; } pz_ray_generator; /* RayGenerator, camera.h:4-41 */
typedef struct pz_lens_params { float distance, thickness, R; } pz_lens_params;   /* LensParams, pk.h:1035-1040 */
typedef struct pz_first_diffuse { pz_float3 p, ng, R; float lambda; } pz_first_diffuse; /* FirstDiffuse, pk.h:80-86 */
/* Texture8RGBX (pk.h:1075-1098): an 8-bit RGBX image (4 bytes per texel, row-major, width x
 * height) in device memory, sampled at the receiver point (x, z) with repeat wrapping and the
 * nearest texel, each channel decoded as (c / 255)^2.2. */
typedef struct pz_texture_rgbx { const uint8_t* texels_dev; uint32_t width, height; } pz_texture_rgbx;
/* RayGenerator::lookat (camera.h:10-22), on the host. */
PZ_API void pz_ray_generator_lookat(pz_ray_generator* gen, pz_float3 eye, pz_float3 center, pz_float3 up, float fovy,
                                    int width, int height);
/* solvePrimary (main_gpu.cu:213-371).  accum_dev: 4 floats per pixel (RGB + sample
 * count), added to.  The albedo of a diffuse hit is the floor texture sampled at the hit's
 * (x, z) as the reference samples it (main_gpu.cu:343), or the constant `albedo` when
 * albedo_texture is NULL; lens->R <= 0 disables the thick lens (pk.h:1042-1073). */
PZ_API int pz_solve_primary(float* accum_dev, pz_first_diffuse* first_diffuse_dev, int width, int height,
                            const pz_ray_generator* gen, const pz_lens_params* lens,
                            const pz_internal_node* internals_dev, const uint32_t* root_dev,
                            const pz_triangle* triangles_dev, const pz_triangle_attrib* attribs_dev, pz_float3 p_light,
                            float light_intensity, float radiance_clamp, float cauchy_a, float cauchy_b,
                            pz_float3 albedo, const pz_texture_rgbx* albedo_texture, int iteration,
                            uint32_t* status_dev, pz_stream_t stream);

/* ---------------------------------------------------------------- (pixel, tuple) work list */
typedef struct pz_specular_path { int32_t pixel; int32_t cache_index; } pz_specular_path; /* pk.h:1102-1106 */
/* lookupFlatten (main_gpu.cu:373-416): appends {pixel, slot} and {path hash, index}
 * (IndexedSpecularPath as u64: hash in bits 0..31) for every slot of each pixel's cell
 * with the given event descriptor; *counter_dev (device) is the running count and must
 * be zeroed by the caller.  Pixels whose entries would pass `capacity` are dropped and
 * flagged in the cache status word. */
PZ_API int pz_lookup_flatten(uint32_t events, pz_specular_path* paths_dev, uint64_t* indexed_dev,
                             uint32_t* counter_dev, uint32_t capacity, const pz_first_diffuse* first_diffuse_dev,
                             int n_pixels, void* cache_dev, uint32_t cache_capacity, float cell_step,
                             pz_stream_t stream);
/* reorderSpecularPath (main_gpu.cu:515-525): dst[i] = src[indexed[i] >> 32]. */
PZ_API int pz_reorder_specular_paths(const uint64_t* indexed_dev, pz_specular_path* dst_dev,
                                     const pz_specular_path* src_dev, uint32_t n, pz_stream_t stream);

/* ---------------------------------------------------------------- specular solve
 * Description of one specular solve over a work list (solveSpecularPath<K>,
 * main_gpu.cu:418-486).  Reference mode (spectral == NULL): each item uses its pixel's
 * sampled wavelength and adds RGB to accum (4 floats per pixel).  Binned mode
 * (spectral != NULL): each (item, bin) uses etas[bin] and adds the clamped contribution
 * to spectral[pixel * n_bins + bin]. */
typedef struct pz_solve_desc {
    int K;                                 /* chain length, 1..4 */
    uint32_t events;                       /* EventDescriptor::asU32 (pk.h:156-158) */
    const pz_specular_path* paths;         /* device work list */
    uint64_t n_paths;
    const pz_first_diffuse* first_diffuse; /* device, per pixel */
    const pz_internal_node* internals;
    const uint32_t* root;
    const pz_triangle* triangles;
    const pz_triangle_attrib* attribs;
    void* cache;
    uint32_t cache_capacity;
    float cell_step;
    pz_float3 p_light;
    float light_intensity;                 /* 16 in the reference (pk.h:1686) */
    float radiance_clamp;                  /* 12 (pk.h:1688) */
    float cauchy_a, cauchy_b;              /* eta(lambda) = a + b / lambda^2, lambda in nm */
    float* accum;
    float* spectral;
    const float* etas;                     /* device, n_bins */
    int n_bins;
    int max_iterations;                    /* 32 (main_gpu.cu:456) */
    float cost_tolerance;                  /* 1e-10 */
    int early_term_warmup;                 /* 1 */
    unsigned long long* stats;             /* device u64[3]: items solved, converged, contributing (or NULL) */
    int fma_contraction;                   /* plain solve: 0 (the default) = no FMA contraction, the reference's float
                                              arithmetic of the CPU code bit for bit; 1 = contracted multiply-adds
                                              (faster, but edge and fold decisions move: about 4e-3 relative RMSE
                                              on the dispersive-sphere image) */
    float polish_det;                      /* batched solve: FP64 polish of roots whose relative determinant
                                              prod|R_ii| / max|R_ii|^(2K) is below this; <= 0 = never (the
                                              default: the image then follows the reference's float
                                              arithmetic); 1e-6 polishes near-singular Jacobians */
    int continuation;                      /* batched solve: 1 = refine each bin from its predicted root
                                              (faster; roots near triangle edges are accepted more often
                                              than the reference's Newton path accepts them) */
    float fold_det;                        /* batched solve: items whose roots have a relative determinant
                                              below this (near a fold of the caustic) are solved bin by bin
                                              from the photon barycentrics; 0 = 1e-2, < 0 = never */
    float graze_cos;                       /* batched solve: roots where a path segment meets a surface at
                                              |cos| below this (near-grazing) are polished in FP64 and
                                              their admissibility is tested in FP64; <= 0 = never (the
                                              default); no reference counterpart */
    float* roots;                          /* optional, NULL = none: the root of every (item, bin) solve that
                                              converged, 8 floats at [(item * n_bins + bin) * 8] (2K used; n_bins
                                              is 1 in reference mode).  Entries of bins that were not solved or
                                              did not converge are left as they were: fill the buffer with NaN
                                              first to tell them apart.  The batched solve solves only the bins
                                              that can contribute (a bin whose root lies outside a triangle is
                                              skipped) */
} pz_solve_desc;
/* One thread per work item, one launch per call: the reference's plain structure. */
PZ_API int pz_solve_specular_plain(const pz_solve_desc* desc, pz_stream_t stream);

/* Batched persistent solve (binned mode only, n_bins <= 64): the same work items and
 * per-bin semantics as pz_solve_specular_plain, scheduled for the GPU -- persistent
 * warps, the root of every bin predicted from one centre-bin solve and its derivative
 * in eta, bins outside the triangles rejected without a solve, warp-shared visibility
 * queries, FP64 polish of ill-conditioned roots.  n_paths_dev (device u32, e.g. the
 * lookup counter) gives the item count on the device so no host round trip is needed
 * (desc->n_paths is then the capacity); NULL uses desc->n_paths.  blocks_per_sm <= 0
 * picks the default.  scratch: pz_solve_batched_scratch_bytes(K, capacity, n_bins) bytes (0 for
 * K outside 1..4 or n_bins outside 1..64). */
PZ_API size_t pz_solve_batched_scratch_bytes(int K, uint64_t max_paths, int n_bins);
/* After a batched solve: the scratch header holds u64 diagnostics at byte offset 64:
 * items skipped by prediction, predicted, plain fallback, per-bin Newton solves, FP64
 * polishes, visibility-query overflows, visibility candidates, visibility queries,
 * fallbacks because the centre solve did not converge, fallbacks of items whose branch
 * converged (near a fold, or a predicted shift over the band too large), fallbacks because a
 * probe disagreed with the predicted branch, phase-2 Newton iterations, phase-2 bins refined
 * from a predicted root, fallbacks near a fold (relative det below fold_det; part of the
 * converged-branch fallbacks). */
PZ_API int pz_solve_specular_batched(const pz_solve_desc* desc, const uint32_t* n_paths_dev, void* scratch_dev,
                                     size_t scratch_bytes, int blocks_per_sm, pz_stream_t stream);

/* Batch of device-side solveConstraints<K> calls (pk.h:466-592) through the device-callable
 * solver of palzilla_b200_device.cuh, one per item, in the reference's float arithmetic (no
 * FMA contraction: equal to its CPU code bit for bit).  Item i solves the chain of triangles
 * tuples_dev[i*K .. i*K+K) (indices into triangles_dev / attribs_dev) from p_beg to
 * p_end_dev[i] at eta etas_dev[i], starting from the 2K barycentrics params_dev[i*2K ..],
 * which are overwritten with the solver's last iterate (the root when it converged).
 * converged_dev[i] (may be NULL) = 1 when the cost tolerance was reached; iters_dev[i] (may
 * be NULL) = the last iteration passed to the end-of-iteration callback (-1 when the solve
 * was rejected at a triangle edge before any callback).  An item whose triangle indices are
 * not below n_triangles is not solved: converged 0, iteration -2, parameters unchanged. */
PZ_API int pz_solve_constraints(int K, uint32_t events, pz_float3 p_beg, const int32_t* tuples_dev,
                                const pz_float3* p_end_dev, const float* etas_dev, uint32_t n,
                                const pz_triangle* triangles_dev, const pz_triangle_attrib* attribs_dev,
                                uint32_t n_triangles, int max_iterations, float cost_tolerance, int early_term_warmup, float* params_dev,
                                uint8_t* converged_dev, int32_t* iters_dev, pz_stream_t stream);

/* ---------------------------------------------------------------- batches of scenes
 * No reference counterpart.  Many scenes (each with its own triangles, BVH, PathCache,
 * eye pass, work list and spectral image; one K and one bin count for all) solved by the
 * batched persistent solver in one set of launches: one device work queue over the
 * concatenated work items of every scene, each item solving in its own scene.
 * pz_solve_multi_prepare uploads the scene table into the scratch (synchronises the
 * stream: do it before any stream capture); n_paths_dev[i] is scene i's device item count
 * (e.g. its lookup counter; NULL entries or a NULL array: descs[i].n_paths), descs[i].n_paths
 * its capacity.  pz_solve_specular_multi then only enqueues work (memsets and kernels), so
 * a frame that calls it can be captured in a CUDA graph.  Tuning: probe / phase-1 blocks per
 * SM, phase-2 blocks per SM (1 or 2), and records a phase-2 warp claims per queue access
 * (1..8); NULL = the best found by pz_solve_multi_autotune for this (K, bins, capacity),
 * else {8, 2, 4}.
 * pz_solve_multi_autotune renders the batch once per candidate (clear the images after
 * it) and keeps the fastest. */
typedef struct pz_batch_tuning { int p1_blocks_per_sm, p2_blocks_per_sm, p2_chunk; } pz_batch_tuning;
PZ_API size_t pz_solve_multi_scratch_bytes(int K, int n_bins, uint32_t n_scenes, uint64_t max_paths_total);
PZ_API int pz_solve_multi_prepare(const pz_solve_desc* descs, const uint32_t* const* n_paths_dev, uint32_t n_scenes,
                                  void* scratch_dev, size_t scratch_bytes, pz_stream_t stream);
PZ_API int pz_solve_specular_multi(int K, int n_bins, uint32_t n_scenes, uint64_t max_paths_total, void* scratch_dev,
                                   size_t scratch_bytes, const pz_batch_tuning* tuning, unsigned long long* stats_dev,
                                   pz_stream_t stream);
PZ_API int pz_solve_multi_autotune(int K, int n_bins, uint32_t n_scenes, uint64_t max_paths_total, void* scratch_dev,
                                   size_t scratch_bytes, unsigned long long* stats_dev, pz_batch_tuning* best_out,
                                   float* best_ms_out, pz_stream_t stream);

/* ---------------------------------------------------------------- Path Cuts
 * InternalNormalBound (pk.h:1705-1709, 52 B): for each internal node, the bounds of the
 * shading normals of the triangles under each child. */
typedef struct pz_normal_bound { pz_aabb normal_bounds[2]; uint32_t counter; } pz_normal_bound;
/* Normal bounds of a BVH from pz_bvh_build (main.cpp:250-295), for its n_internals nodes. */
PZ_API int pz_normal_bounds(const pz_internal_node* internals_dev, int n_internals,
                            const pz_triangle_attrib* attribs_dev, pz_normal_bound* out_dev, pz_stream_t stream);
/* Scratch for pz_path_cuts: a 256-byte header and two frontiers of frontier_capacity node
 * tuples (at least n_queries; more lets wider trees through). */
PZ_API size_t pz_path_cuts_scratch_bytes(int K, uint32_t frontier_capacity);
/* Replaces traverseAdmissibleNodes<K> (pk.h:1760-2220) for a batch of queries: every
 * admissible K-triangle tuple of the event chain `events` from p_beg to each p_end_dev[q],
 * found by interval culling over BVH node tuples (BVH built with
 * PZ_BUILD_OPTION_USE_NORMAL in the reference's use).  Writes (1 + K) u32 per tuple
 * {q, triangle[0..K)} to tuples_dev (unordered), and the tuple count (which may exceed
 * tuple_capacity: PZ_ERR_DEVICE is then returned) to *n_tuples_out, and the number of
 * node tuples tested to *node_tuples_out (may be NULL).  directed_rounding = 0 runs the
 * reference's round-to-nearest arithmetic (the same tuple set); 1 rounds every interval
 * bound outward (a superset).  Synchronises `stream` once per tree level. */
PZ_API int pz_path_cuts(int K, uint32_t events, float eta, pz_float3 p_beg, const pz_float3* p_end_dev,
                        uint32_t n_queries, const pz_internal_node* internals_dev, const pz_normal_bound* nbs_dev,
                        const pz_triangle* triangles_dev, const pz_triangle_attrib* attribs_dev,
                        const uint32_t* root_dev, int directed_rounding, uint32_t* tuples_dev, uint32_t tuple_capacity,
                        uint64_t* n_tuples_out, uint64_t* node_tuples_out, void* scratch_dev, size_t scratch_bytes,
                        pz_stream_t stream);

/* ---------------------------------------------------------------- subdivision solve
 * No reference counterpart (the reference solves each admissible tuple once, from one
 * start: main.cpp:1052).  For every tuple row {q, triangle[0..K)} -- the rows pz_path_cuts
 * writes -- the domain of the 2K barycentrics is bisected (split t halves dimension
 * t mod 2K) under affine bounds of the specular constraint of solveConstraints<K>
 * (pk.h:466-592) with rounding-error terms rounded upward; boxes whose bound excludes
 * zero, that lie outside a triangle or whose cosines rule the event out are dropped.
 * A box stops splitting at max_depth, or when every bounded residual component is
 * narrower than eps; its centre starts the Newton solve for each wavelength bin
 * (eta = etas_dev[bin]; the bins share one subdivision, with eta^2 - 1 as one more noise
 * symbol) whose residual, with that bin's eta substituted, may vanish in the box.  A root is kept when it
 * converged, lies in its own box (each root has one owner box) and
 * contributableThroughput (pk.h:760-842) is positive.  The tuple rows index
 * triangles_dev / attribs_dev (the specular soup pz_path_cuts ran on, or the scene);
 * visibility runs through the scene's BVH (scene_internals_dev, scene_triangles_dev,
 * scene_root_dev). */
typedef struct pz_subdiv_params {
    int max_depth;         /* 12: bisections of a tuple's domain (0..20) */
    float eps;             /* 1e-4: residual width at which a box stops splitting */
    int max_iterations;    /* 32 (main_gpu.cu:456) */
    float cost_tolerance;  /* 1e-10 */
    int early_term_warmup; /* 1 */
    int fp64_polish;       /* 0; 1 = 4 FP64 Newton steps on every root found in its box */
} pz_subdiv_params;
typedef struct pz_subdiv_stats {
    uint64_t boxes_tested, boxes_culled, leaves;
    uint64_t bins_excluded; /* (leaf, bin) pairs whose residual for that bin excludes zero */
    uint64_t solves, converged, outside_box, roots, polished;
} pz_subdiv_stats;
typedef struct pz_specular_root {
    uint32_t tuple;   /* row of tuples_dev */
    uint32_t bin;     /* wavelength bin */
    uint32_t depth;   /* owner box: depth ... */
    uint32_t path;    /* ... and bisection path (bit t = half taken at split t) */
    float params[8];  /* barycentrics (u, v) per vertex; 2K used */
    float throughput; /* contributableThroughput, > 0 */
    uint32_t pad[3];
} pz_specular_root;   /* 64 bytes */
/* Scratch: a 256-byte header, a box queue of 2 * box_capacity entries and the leaf list of
 * box_capacity entries (box_capacity >= n_tuples).  All depths are bounded in one persistent
 * kernel: each warp keeps the boxes of its tuples on a stack in shared memory and the queue
 * (a ring in the scratch) holds the tuples, the boxes a stack cannot take and the boxes
 * lent to idle warps, so it needs little room; the leaf list must hold every leaf.  The
 * queue's space then holds the (leaf, bin) solve list (2 * box_capacity entries). */
PZ_API size_t pz_subdivide_scratch_bytes(uint64_t box_capacity);
/* Writes the kept roots (unordered) to roots_dev and their count (which may exceed
 * root_capacity: PZ_ERR_DEVICE is then returned) to *n_roots_out.  Synchronises `stream`
 * twice: for the leaf count (the leaves are sorted by tuple row before they are solved)
 * and at the end. */
PZ_API int pz_subdivide_solve(int K, uint32_t events, pz_float3 p_beg, const pz_float3* p_end_dev,
                              const uint32_t* tuples_dev, uint32_t n_tuples, const float* etas_dev, int n_bins,
                              const pz_subdiv_params* params, const pz_triangle* triangles_dev,
                              const pz_triangle_attrib* attribs_dev, const pz_internal_node* scene_internals_dev,
                              const pz_triangle* scene_triangles_dev, const uint32_t* scene_root_dev,
                              pz_specular_root* roots_dev, uint64_t root_capacity, uint64_t* n_roots_out,
                              pz_subdiv_stats* stats_out, void* scratch_dev, size_t scratch_bytes,
                              pz_stream_t stream);
/* The roots' contributions to a binned spectral image (spectral_dev: n_pixels x n_bins
 * floats, accumulated): the tail of solveSpecularPath<K> (main_gpu.cu:466-486) with the
 * wavelength fixed to each root's bin -- throughput * light_intensity / dAdw * cos at the
 * receiver, clamped at radiance_clamp.  The tuple rows' query index is the pixel of
 * first_diffuse_dev (pz_solve_primary's FirstDiffuse records; the solve's p_end of a
 * query is that pixel's receiver point).  Triangles as for pz_subdivide_solve. */
PZ_API int pz_subdivide_contribute(int K, uint32_t events, pz_float3 p_beg, float light_intensity,
                                   float radiance_clamp, const uint32_t* tuples_dev,
                                   const pz_specular_root* roots_dev, uint64_t n_roots, const void* first_diffuse_dev,
                                   const float* etas_dev, int n_bins, const pz_triangle* triangles_dev,
                                   const pz_triangle_attrib* attribs_dev, float* spectral_dev, pz_stream_t stream);

/* ---------------------------------------------------------------- adjoint
 * No reference counterpart.  A forward / backward pair for gradients of a loss on the
 * binned spectral image.  Forward: the plain binned solve in the reference's arithmetic
 * (fma_contraction is ignored) into desc->spectral.  Backward (same descriptor and work
 * list, geometry unchanged since the forward): recomputes each path's root from the
 * photon's barycentrics, and for every accepted, unclamped path adds
 * dL/dI[pixel][bin] * dI/dp to the gradients, by the implicit-function theorem at the
 * root: grad_heights_dev[v] += dL/d(y of vertex v) through corner_vertex_dev (3 int32 per
 * triangle: the vertex whose height is that corner's y, or -1), grad_cauchy_dev[0..1] +=
 * dL/dA, dL/dB of eta = A + B / lambda^2.  The gradient arrays accumulate (clear them
 * first).  K = 1 or 2. */
PZ_API int pz_adjoint_forward(const pz_solve_desc* desc, pz_stream_t stream);
PZ_API int pz_adjoint_backward(const pz_solve_desc* desc, const float* dloss_dspectral_dev,
                               const int32_t* corner_vertex_dev, float* grad_heights_dev, float* grad_cauchy_dev,
                               pz_stream_t stream);
/* The same gradients as pz_adjoint_backward (up to the order of the float atomics), in two
 * kernels: one keeps the accepted, unclamped (path, bin) pairs and their roots in a list
 * in scratch_dev (a 256-byte header and 32 bytes per pair, pz_adjoint_scratch_bytes(
 * capacity)), the other differentiates only those.  Pairs beyond the capacity are dropped
 * and set PZ_DEVICE_ERR_CAPACITY in the scratch status word (pz_scratch_status).  Does not
 * synchronise. */
PZ_API size_t pz_adjoint_scratch_bytes(uint64_t capacity);
PZ_API int pz_adjoint_backward_compact(const pz_solve_desc* desc, const float* dloss_dspectral_dev,
                                       const int32_t* corner_vertex_dev, float* grad_heights_dev,
                                       float* grad_cauchy_dev, void* scratch_dev, size_t scratch_bytes,
                                       pz_stream_t stream);

/* ---------------------------------------------------------------- resolve
 * pack (main_gpu.cu:499-513): accumulator / count -> sRGB OETF -> RGBA8. */
PZ_API int pz_resolve(uint32_t* pixels_dev, const float* accum_dev, int n_pixels, pz_stream_t stream);
/* Spectral image -> linear sRGB (rgb_dev, 4 floats per pixel, may be NULL) and RGBA8
 * (pixels_dev, may be NULL): (albedo/pi) * sum_b S_b * srgb(lambda_b) * dlambda. */
PZ_API int pz_resolve_spectral(float* rgb_dev, uint32_t* pixels_dev, const float* spectral_dev, int n_pixels,
                               int n_bins, float lambda_min, float lambda_max, pz_float3 albedo, pz_stream_t stream);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* PALZILLA_B200_H */
