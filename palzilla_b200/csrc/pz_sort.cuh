// pz_sort.cuh -- onesweep LSD radix sort for sm_100a (8-bit digits).
//
// Behaviour of the reference sorter (tinyhiponesweep.h:592-668): a stable sort of
// 32- or 64-bit keys on digit passes covering bits [startBit, startBit + 8 *
// ceil((endBit - startBit) / 8)), optionally carrying a u32 value per key, with the
// result ending in the caller's buffers.  Each digit is the full 8 bits at its
// position (tinyhiponesweep.h:93-94), so a partial last digit also orders on the
// bits above endBit, exactly as the reference does.
//
// Design (independent of the reference's kernels):
//  * one histogram kernel computes every pass's digit counts in a single read and,
//    in the same launch, clears the look-back table;
//  * one kernel per pass: tiles of kThreads x kItems items claim a tile index from an
//    atomic counter (so a tile only ever waits on tiles that are already running), count
//    digits per warp and publish the tile's aggregate before ranking, rank keys stably
//    from per-warp digit masks in shared memory, resolve the tile's global digit offsets
//    with a decoupled look-back over 64-bit words {value, flag, pass tag} that loads
//    kLookBatch predecessors at a time, stage the tile in shared memory in digit order and
//    write digit runs out coalesced;
//  * every spin wait is bounded; on expiry the kernel sets kErrSpinLimit in the
//    status word and finishes (with undefined output) instead of hanging.
#pragma once
#include "pz_common.cuh"

namespace pz {
namespace sort {

// Compile-time shape of the digit pass: threads per tile, items per thread, ranking by
// warp ballots (0), match.any (1) or lane bits OR-ed into per-warp digit masks in shared
// memory (2, with early counts only), digit counts before ranking (1) or from the
// ranking (0), minimum blocks per SM.  Sweeps on 2^24 64-bit keys (4 digit passes, L2
// flushed, median of 7) chose the defaults: masks in shared memory, 20 items, 3 blocks
// (0.460 ms); the best ballot shape took 0.478 ms, 16 items with 4 blocks 0.482 ms, and
// match.any 0.726 ms.  Override them through the build (PZ_EXTRA_NVCC_FLAGS).
#ifndef PZ_SORT_THREADS
#define PZ_SORT_THREADS 256
#endif
#ifndef PZ_SORT_ITEMS
#define PZ_SORT_ITEMS 20
#endif
#ifndef PZ_SORT_RANK_MATCH
#define PZ_SORT_RANK_MATCH 2
#endif
#ifndef PZ_SORT_EARLY_COUNTS
#define PZ_SORT_EARLY_COUNTS 1
#endif
#ifndef PZ_SORT_MIN_BLOCKS
#define PZ_SORT_MIN_BLOCKS 3
#endif
constexpr int kThreads = PZ_SORT_THREADS;
constexpr int kWarps = kThreads / 32;
constexpr int kItems = PZ_SORT_ITEMS;
constexpr int kRankMode = PZ_SORT_RANK_MATCH;
constexpr bool kEarlyCounts = PZ_SORT_EARLY_COUNTS != 0;
constexpr int kMinBlocks = PZ_SORT_MIN_BLOCKS;
constexpr int kTile = kThreads * kItems;  // items per tile
constexpr int kRadix = 256;
constexpr int kMaxPasses = 8;
constexpr int kHistBlocksPerSM = 4;
constexpr uint32_t kSpinLimit = 1u << 22;
#ifndef PZ_SORT_LOOK_BATCH
#define PZ_SORT_LOOK_BATCH 8
#endif
constexpr int kLookBatch = PZ_SORT_LOOK_BATCH;  // predecessor words a look-back step loads at once

// Scratch header (the first kHeaderBytes of the sort scratch).
struct Header {
    uint32_t status;                       // kErr* bits
    uint32_t pad0[31];
    uint32_t tile_counter[kMaxPasses];
    uint32_t pad1[32 - kMaxPasses];
    uint32_t hist[kMaxPasses][kRadix];     // digit counts per pass
};
constexpr size_t kHeaderBytes = 16384;
static_assert(sizeof(Header) <= kHeaderBytes, "header");
// The digit stage runs one thread per digit, and warps are whole.
static_assert(kThreads >= kRadix && kThreads % 32 == 0, "PZ_SORT_THREADS: a multiple of 32, at least 256");
// Per-item ranks within a tile are kept as uint16.
static_assert(kTile <= 65536, "PZ_SORT_THREADS * PZ_SORT_ITEMS must not exceed 65536");

inline uint32_t num_tiles(uint32_t n) { return (n + kTile - 1) / kTile; }
inline int num_passes(int startBit, int endBit) { return (endBit - startBit + 7) / 8; }
inline size_t lookback_bytes(uint32_t n) { return (size_t)num_tiles(n) * kRadix * sizeof(unsigned long long); }
inline size_t scratch_bytes(uint32_t n) { return kHeaderBytes + ((lookback_bytes(n) + 255) & ~(size_t)255); }

// Launch helpers (defined in pz_sort.cu).  `hist_done` means the histogram and the
// look-back clear were already produced by a fused producer (the Morton kernel).
template <class KeyT>
cudaError_t launch_hist(const KeyT* keys, uint32_t n, int startBit, int nPasses, Header* h,
                        unsigned long long* lookback, cudaStream_t s);
template <class KeyT>
cudaError_t launch_passes(KeyT* keys, uint32_t* vals, KeyT* tmpKeys, uint32_t* tmpVals, uint32_t n, int startBit,
                          int nPasses, Header* h, unsigned long long* lookback, cudaStream_t s);

// Device helpers shared with fused producers.
template <class KeyT>
PZ_D uint32_t digit_of(KeyT k, int bit) { return (uint32_t)(k >> bit) & 0xFFu; }

// Clears `words` 64-bit look-back entries with a grid-stride loop (16-byte stores).
PZ_D void clear_lookback(unsigned long long* lb, size_t words)
{
    size_t pairs = words / 2;
    uint4* p = reinterpret_cast<uint4*>(lb);
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < pairs; i += (size_t)gridDim.x * blockDim.x)
        p[i] = make_uint4(0, 0, 0, 0);
}

}  // namespace sort
}  // namespace pz
