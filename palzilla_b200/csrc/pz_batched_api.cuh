// pz_batched_api.cuh -- batched persistent solver interface (see pz_batched.cu).
#pragma once
#include "pz_solve.cuh"

namespace pz {
namespace batched {

struct BatchArgs {
    SolveArgs s;                       // binned mode only (s.spectral, s.etas, s.nBins <= 64)
    const uint32_t* nPathsDev;         // device item count (the lookup counter), or null: s.nPaths
    unsigned long long* workCounter;   // device scratch word (zeroed by the launcher)
    unsigned long long* recordCount;   // device scratch word (zeroed by the launcher)
    void* records;                     // phase-1 records, recordCapacity of record_bytes(K)
    unsigned long long recordCapacity;
    void* probes;                      // plain-solve probes, 3 per work item of probe_bytes(K), s.nPaths items
    uint32_t* status;                  // status word (capacity overflow)
    unsigned long long* counters;      // device u64[kNumCounters] diagnostics (see kCnt*), or null
    double polishDet;                  // FP64 polish below this relative det (<= 0: never)
    int continuation;                  // 1: refine predicted roots instead of solving from the photon start
    float illDet;                      // relative det below which an item takes per-bin solves (near a fold)
};

// diagnostics counters
enum {
    kCntMode0 = 0, kCntMode1, kCntMode2, kCntNewton2, kCntPolish, kCntFatOverflow, kCntCandidates, kCntQueries,
    kCntFallbackNoConv, kCntFallbackShift, kCntFallbackProbe, kNumCounters
};

// bytes of one phase-1 record for chain length K
size_t record_bytes(int K);
// bytes of one plain-solve probe (root and verdict) for chain length K
size_t probe_bytes(int K);
cudaError_t launch_solve_batched(int K, const BatchArgs& a, int blocksPerSM, cudaStream_t s);

}  // namespace batched
}  // namespace pz
