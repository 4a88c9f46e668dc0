// pz_batched_api.cuh -- batched persistent solver interface (see pz_batched.cu).
#pragma once
#include "pz_solve.cuh"

namespace pz {
namespace batched {

struct SceneArgs;

struct BatchArgs {
    SolveArgs s;                       // binned mode only (s.spectral, s.etas, s.nBins <= 64)
    const uint32_t* nPathsDev;         // device item count (the lookup counter), or null: s.nPaths
    unsigned long long* workCounter;   // device scratch word (zeroed by the launcher)
    unsigned long long* recordCount;   // device scratch word (zeroed by the launcher)
    // Records of items solved bin by bin (every bin from the photon's start) form a second
    // queue, filled from the end of the records array; each item makes at most one record and
    // the capacity covers every item, so the two queues never meet.
    unsigned long long* workCounter2;  // device scratch word (zeroed by the launcher)
    unsigned long long* recordCount2;  // device scratch word (zeroed by the launcher)
    void* records;                     // phase-1 records, recordCapacity of record_bytes(K)
    unsigned long long recordCapacity;
    void* probes;                      // plain-solve probes, 3 per work item of probe_bytes(K), s.nPaths items
    uint32_t* status;                  // status word (capacity overflow)
    unsigned long long* counters;      // device u64[kNumCounters] diagnostics (see kCnt*), or null
    double polishDet;                  // FP64 polish below this relative det (<= 0: never)
    float grazeCos = 0.0f;             // FP64 polish and admissibility below this |cos| (<= 0: never)
    int continuation;                  // 1: refine predicted roots instead of solving from the photon start
    float illDet;                      // relative det below which an item takes per-bin solves (near a fold)
    int chunk = 0;                     // records a phase-2 warp claims per queue access (0: kP2ChunkDefault)
    const SceneArgs* scenes = nullptr; // batch of scenes (device table), or null: the single scene s
    uint32_t nScenes = 0;
    const unsigned long long* offsets = nullptr;  // nScenes + 1 item offsets of the batch
    // phase 2: accepted roots and their per-round blocks, reused by every wave
    void* accepted = nullptr;          // acceptCapacity entries of accepted_bytes(K)
    unsigned long long acceptCapacity = 0;
    void* blocks = nullptr;            // blockCapacity entries of block_bytes()
    unsigned long long blockCapacity = 0;
    unsigned long long* p2 = nullptr;  // device u64[4] (scratch header byte 192): accepted count, block count,
                                       // reserved, blocks taken
    int wave = 0;                      // phase-2 wave of this launch (0 .. kMaxWaves - 1)
};

// Phase 2 runs in at most kMaxWaves waves; each wave has room for nBins accepted roots (a
// record's most) per record of 1/kMaxWaves of the record capacity, so every record fits.
constexpr int kMaxWaves = 8;
// blocks per SM the phase-1 and phase-2 solve kernels are built for (register budget)
#ifndef PZ_P2_SOLVE_BLOCKS
#define PZ_P2_SOLVE_BLOCKS 2
#endif
#ifndef PZ_PHASE1_BLOCKS
#define PZ_PHASE1_BLOCKS 2
#endif
constexpr int kP2SolveBlocks = PZ_P2_SOLVE_BLOCKS;
constexpr int kPhase1Blocks = PZ_PHASE1_BLOCKS;
// Relative determinant of an item's branch of roots below which the item is solved bin by bin
// (near a fold of the caustic, where the prediction of the bins' roots is least reliable).
constexpr float kDefaultFoldDet = 1.0e-2f;
// Phase-2 warps claim records in chunks of up to kP2ChunkMax (kP2ChunkDefault unless a tuning
// says otherwise); a wave's room is padded by one chunk so that it still takes its share of
// the records when its last reservations are for whole chunks.
#ifndef PZ_P2_CHUNK
#define PZ_P2_CHUNK 4
#endif
constexpr int kP2ChunkMax = 8;
constexpr int kP2ChunkDefault = PZ_P2_CHUNK;
static_assert(kP2ChunkDefault >= 1 && kP2ChunkDefault <= kP2ChunkMax, "PZ_P2_CHUNK: 1..8");
inline unsigned long long wave_records(unsigned long long recordCapacity)
{
    return (recordCapacity + kMaxWaves - 1) / kMaxWaves + kP2ChunkMax;
}
inline unsigned long long accept_capacity(unsigned long long recordCapacity, int nBins)
{
    return (unsigned long long)nBins * wave_records(recordCapacity);
}
// at most three rounds (blocks) per record: B <= 64 bins on consecutive lanes of 32-lane
// rounds that other records' bins may start and end
inline unsigned long long block_capacity(unsigned long long recordCapacity)
{
    return 3ull * wave_records(recordCapacity);
}

// One scene of a batch: its solve arguments and its item count on the device.
struct SceneArgs {
    SolveArgs s;
    const uint32_t* nPathsDev;         // or null: s.nPaths
};

// diagnostics counters
enum {
    kCntMode0 = 0, kCntMode1, kCntMode2, kCntNewton2, kCntPolish, kCntFatOverflow, kCntCandidates, kCntQueries,
    kCntFallbackNoConv, kCntFallbackShift, kCntFallbackProbe, kCntNewtonIters, kCntWarm, kCntFallbackFold, kNumCounters
};

// bytes of one phase-1 record for chain length K
size_t record_bytes(int K);
// bytes of one accepted phase-2 root, and of one block of them
size_t accepted_bytes(int K);
size_t block_bytes();
// bytes of one plain-solve probe (root and verdict) for chain length K
size_t probe_bytes(int K);
cudaError_t launch_solve_batched(int K, const BatchArgs& a, int blocksPerSM, cudaStream_t s);
// Batch of scenes: item offsets (one small kernel) then the same three launches; the
// tuning picks the probe / phase-1 grid (blocks per SM) and phase 2's blocks per SM.
cudaError_t launch_solve_batched_multi(int K, const BatchArgs& a, int p1BlocksPerSM, int p2BlocksPerSM,
                                       unsigned long long* offsets, cudaStream_t s);

}  // namespace batched
}  // namespace pz
