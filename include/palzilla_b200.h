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

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* PALZILLA_B200_H */
