// pz_sort.cu -- onesweep radix sort kernels (see pz_sort.cuh for the design).
#include "pz_sort.cuh"

namespace pz {
namespace sort {

// ---------------------------------------------------------------------------
// histogram of every digit pass + look-back clear
// ---------------------------------------------------------------------------
template <class KeyT>
__global__ void __launch_bounds__(kThreads) k_hist(const KeyT* __restrict__ keys, uint32_t n, int startBit,
                                                   int nPasses, Header* __restrict__ h, unsigned long long* lookback,
                                                   size_t lookbackWords)
{
    __shared__ uint32_t sh[kMaxPasses * kRadix];
    for (int i = threadIdx.x; i < nPasses * kRadix; i += kThreads) sh[i] = 0;
    __syncthreads();
    clear_lookback(lookback, lookbackWords);

    constexpr int kPerVec = 16 / sizeof(KeyT);
    const uint32_t nVec = (reinterpret_cast<uintptr_t>(keys) & 15) ? 0u : n / kPerVec;
    const uint4* v4 = reinterpret_cast<const uint4*>(keys);
    const uint32_t stride = gridDim.x * kThreads;
    for (uint32_t i = blockIdx.x * kThreads + threadIdx.x; i < nVec; i += stride) {
        uint4 q = __ldcs(v4 + i);
        KeyT k[kPerVec];
        memcpy(k, &q, 16);
#pragma unroll
        for (int e = 0; e < kPerVec; e++)
            for (int p = 0; p < nPasses; p++) atomicAdd(&sh[p * kRadix + digit_of(k[e], startBit + 8 * p)], 1u);
    }
    for (uint32_t i = nVec * kPerVec + blockIdx.x * kThreads + threadIdx.x; i < n; i += stride) {
        KeyT k = keys[i];
        for (int p = 0; p < nPasses; p++) atomicAdd(&sh[p * kRadix + digit_of(k, startBit + 8 * p)], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nPasses * kRadix; i += kThreads) {
        uint32_t c = sh[i];
        if (c) atomicAdd(&h->hist[0][0] + i, c);
    }
}

// ---------------------------------------------------------------------------
// one digit pass
// ---------------------------------------------------------------------------
constexpr unsigned long long kFlagA = 1ull << 32;  // tile aggregate published
constexpr unsigned long long kFlagP = 2ull << 32;  // inclusive prefix published

PZ_D unsigned long long ld_volatile(const unsigned long long* p)
{
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
PZ_D void st_volatile(unsigned long long* p, unsigned long long v)
{
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Exclusive block-wide scan of one value per thread (256 threads); returns the
// exclusive prefix.  `ws` is kWarps words of shared scratch.
PZ_D uint32_t block_exclusive_scan(uint32_t x, uint32_t* ws)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t inc = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xFFFFFFFFu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) ws[warp] = inc;
    __syncthreads();
    uint32_t wpre = 0;
#pragma unroll
    for (int w = 0; w < kWarps; w++) wpre += (w < warp) ? ws[w] : 0u;
    __syncthreads();
    return wpre + inc - x;
}

static_assert(kRankMode != 2 || kEarlyCounts, "ranking mode 2 needs early counts");

template <class KeyT, bool kHasVal>
struct PassSmem {
    KeyT keys[kTile];                 // tile in digit order
    uint32_t vals[kHasVal ? kTile : 1];
    uint32_t off[kWarps][kRadix];     // per-warp digit counts, then per-warp positions
    uint32_t match[kRankMode == 2 ? kWarps : 1][kRadix];  // per-warp lane masks by digit (ranking mode 2)
    uint32_t gbase[kRadix];           // global destination of the digit run minus its tile start
    uint32_t ws[2][kWarps];
    uint32_t tile;
};

// Peers of this lane: the valid lanes of the warp holding the same digit.
template <bool kAllValid>
PZ_D uint32_t digit_peers(uint32_t d, bool valid)
{
    const uint32_t vmask = kAllValid ? 0xFFFFFFFFu : __ballot_sync(0xFFFFFFFFu, valid);
    if (kRankMode == 1) return __match_any_sync(0xFFFFFFFFu, valid ? d : 0x100u) & vmask;
    uint32_t peers = vmask;
#pragma unroll
    for (int b = 0; b < 8; b++) {
        const bool set = (d >> b) & 1u;
        const uint32_t bal = __ballot_sync(0xFFFFFFFFu, set);
        peers &= set ? bal : ~bal;
    }
    return peers;
}

// One tile of a digit pass; kFull = the tile has kTile items (no per-item bounds checks).
template <class KeyT, bool kHasVal, bool kFull>
PZ_D void pass_tile(PassSmem<KeyT, kHasVal>& S, const KeyT* __restrict__ kin, KeyT* __restrict__ kout,
                    const uint32_t* __restrict__ vin, uint32_t* __restrict__ vout, uint32_t n, int bit, int pass,
                    Header* __restrict__ h, unsigned long long* __restrict__ lookback, uint32_t tile)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t base = tile * kTile;

    // ---- load: warp w owns items [w * 32 * kItems, (w + 1) * 32 * kItems) of the tile,
    //      item k of lane l at offset k * 32 + l (coalesced, and (k, lane) is input order)
    KeyT key[kItems];
    uint32_t val[kHasVal ? kItems : 1];
    const uint32_t wbase = base + warp * (kItems * 32);
#pragma unroll
    for (int k = 0; k < kItems; k++) {
        const uint32_t idx = wbase + k * 32 + lane;
        if (kFull || idx < n) {
            key[k] = __ldcs(kin + idx);
            if (kHasVal) val[k] = __ldcs(vin + idx);
        } else {
            key[k] = 0;
            if (kHasVal) val[k] = 0;
        }
    }

    // ---- per-warp digit counts: either counted up front (the tile aggregate can then be
    //      published before ranking) or produced by the ranking itself
    uint16_t rank[kEarlyCounts ? 1 : kItems];
    const uint32_t ltmask = (1u << lane) - 1u;
    if (kEarlyCounts) {
#pragma unroll
        for (int k = 0; k < kItems; k++)
            if (kFull || wbase + k * 32 + lane < n) atomicAdd(&S.off[warp][digit_of(key[k], bit)], 1u);
    } else {
#pragma unroll
        for (int k = 0; k < kItems; k++) {
            const bool valid = kFull || wbase + k * 32 + lane < n;
            const uint32_t dd = digit_of(key[k], bit);
            const uint32_t peers = digit_peers<kFull>(dd, valid);
            const uint32_t before = __popc(peers & ltmask);
            const uint32_t cnt = valid ? S.off[warp][dd] : 0u;
            __syncwarp();
            if (valid && before == 0) S.off[warp][dd] = cnt + __popc(peers);
            __syncwarp();
            rank[k] = (uint16_t)(cnt + before);
        }
    }
    __syncthreads();

    // ---- per digit (thread = digit, kThreads >= kRadix): per-warp positions, tile
    //      total, aggregate published for later tiles
    const int d = tid;
    uint32_t total = 0, dstart = 0, gexcl = 0;
    uint32_t wc[kWarps];
    const unsigned long long tag = (unsigned long long)(pass + 1) << 34;
    unsigned long long* mine = lookback + (size_t)tile * kRadix + (d < kRadix ? d : 0);
    if (d < kRadix) {
#pragma unroll
        for (int w = 0; w < kWarps; w++) {
            wc[w] = S.off[w][d];
            total += wc[w];
        }
        st_volatile(mine, tag | (tile == 0 ? kFlagP : kFlagA) | total);
    }
    const uint32_t gcount = d < kRadix ? h->hist[pass][d] : 0u;
    dstart = block_exclusive_scan(total, S.ws[0]);
    gexcl = block_exclusive_scan(gcount, S.ws[1]);
    if (d < kRadix) {
        uint32_t run = dstart;
#pragma unroll
        for (int w = 0; w < kWarps; w++) {
            S.off[w][d] = run;
            run += wc[w];
        }
    }
    __syncthreads();

    // ---- place every key at its tile position in shared memory (digit order, stable)
#pragma unroll
    for (int k = 0; k < kItems; k++) {
        const bool valid = kFull || wbase + k * 32 + lane < n;
        const uint32_t dd = digit_of(key[k], bit);
        if (kEarlyCounts && kRankMode == 2) {
            // peers: every valid lane sets its bit in the mask of its digit, then reads it;
            // the digit's first lane clears the mask for the next item
            uint32_t* m = S.match[kRankMode == 2 ? warp : 0];
            if (valid) atomicOr(&m[dd], 1u << lane);
            __syncwarp();
            const uint32_t peers = valid ? m[dd] : 0u;
            const uint32_t before = __popc(peers & ltmask);
            const uint32_t run = valid ? S.off[warp][dd] : 0u;
            __syncwarp();
            if (valid) {
                S.keys[run + before] = key[k];
                if (kHasVal) S.vals[run + before] = val[k];
                if (before == 0) {
                    S.off[warp][dd] = run + __popc(peers);
                    m[dd] = 0u;
                }
            }
            __syncwarp();
        } else if (kEarlyCounts) {
            const uint32_t peers = digit_peers<kFull>(dd, valid);
            const uint32_t before = __popc(peers & ltmask);
            const uint32_t run = valid ? S.off[warp][dd] : 0u;
            __syncwarp();
            if (valid) {
                S.keys[run + before] = key[k];
                if (kHasVal) S.vals[run + before] = val[k];
                if (before == 0) S.off[warp][dd] = run + __popc(peers);
            }
            __syncwarp();
        } else if (valid) {
            const uint32_t pos = S.off[warp][dd] + rank[k];
            S.keys[pos] = key[k];
            if (kHasVal) S.vals[pos] = val[k];
        }
    }

    // ---- decoupled look-back over earlier tiles for digit d.  The words of kLookBatch
    //      predecessors are loaded at once (independent loads in flight, each a coalesced row
    //      across the block's digit threads), then consumed in order: aggregates are added up
    //      to the first inclusive prefix; a word not yet published ends the batch, and the
    //      next batch starts at it.  Tile 0 publishes its prefix at once, so every walk ends.
    if (d < kRadix) {
        uint32_t prefix = 0;
        if (tile != 0) {
            int t = (int)tile - 1;
            uint32_t spins = 0;
            bool done = false;
            while (!done) {
                unsigned long long w[kLookBatch];
#pragma unroll
                for (int j = 0; j < kLookBatch; j++)
                    w[j] = t - j >= 0 ? ld_volatile(lookback + (size_t)(t - j) * kRadix + d) : 0ull;
                int used = 0;
#pragma unroll
                for (int j = 0; j < kLookBatch; j++) {
                    if (done || used != j) break;
                    const unsigned long long x = w[j];
                    if ((x & ~0x3FFFFFFFFull) != tag || (x & (3ull << 32)) == 0) break;  // not yet published
                    prefix += (uint32_t)x;
                    used = j + 1;
                    if (x & kFlagP) done = true;
                }
                t -= used;
                if (!done && used == 0) {
                    if (++spins > kSpinLimit) {
                        raise_error(&h->status, kErrSpinLimit);
                        break;
                    }
                    if (spins > 16) __nanosleep(32);
                }
            }
            st_volatile(mine, tag | kFlagP | (uint32_t)(prefix + total));
        }
        S.gbase[d] = gexcl + prefix - dstart;
    }
    __syncthreads();

    // ---- write digit runs to their global positions
    const uint32_t tileN = kFull ? (uint32_t)kTile : min((uint32_t)kTile, n - base);
#pragma unroll 4
    for (uint32_t i = tid; i < tileN; i += kThreads) {
        const KeyT kk = S.keys[i];
        const uint32_t dst = S.gbase[digit_of(kk, bit)] + i;
        if (dst < n) {  // always true unless a look-back wait expired (status already set)
            kout[dst] = kk;
            if (kHasVal) vout[dst] = S.vals[i];
        }
    }
}

template <class KeyT, bool kHasVal>
__global__ void __launch_bounds__(kThreads, kMinBlocks) k_pass(const KeyT* __restrict__ kin, KeyT* __restrict__ kout,
                                                               const uint32_t* __restrict__ vin,
                                                               uint32_t* __restrict__ vout, uint32_t n, int bit,
                                                               int pass, Header* __restrict__ h,
                                                               unsigned long long* __restrict__ lookback)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    auto& S = *reinterpret_cast<PassSmem<KeyT, kHasVal>*>(smem_raw);
    if (threadIdx.x == 0) S.tile = atomicAdd(&h->tile_counter[pass], 1u);
    for (int i = threadIdx.x; i < kWarps * kRadix; i += kThreads) (&S.off[0][0])[i] = 0;
    if (kRankMode == 2)
        for (int i = threadIdx.x; i < kWarps * kRadix; i += kThreads) (&S.match[0][0])[i] = 0;
    __syncthreads();
    const uint32_t tile = S.tile;
    if ((uint64_t)(tile + 1) * kTile <= n)
        pass_tile<KeyT, kHasVal, true>(S, kin, kout, vin, vout, n, bit, pass, h, lookback, tile);
    else
        pass_tile<KeyT, kHasVal, false>(S, kin, kout, vin, vout, n, bit, pass, h, lookback, tile);
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
template <class KeyT>
cudaError_t launch_hist(const KeyT* keys, uint32_t n, int startBit, int nPasses, Header* h,
                        unsigned long long* lookback, cudaStream_t s)
{
    int blocks = num_sms() * kHistBlocksPerSM;
    uint32_t need = (n + kThreads * 8 - 1) / (kThreads * 8);
    if ((uint32_t)blocks > need) blocks = (int)(need > 0 ? need : 1);
    k_hist<KeyT><<<blocks, kThreads, 0, s>>>(keys, n, startBit, nPasses, h, lookback,
                                             (size_t)num_tiles(n) * kRadix);
    return cudaGetLastError();
}

template <class KeyT, bool kHasVal>
static cudaError_t launch_pass(const KeyT* kin, KeyT* kout, const uint32_t* vin, uint32_t* vout, uint32_t n, int bit,
                               int pass, Header* h, unsigned long long* lookback, cudaStream_t s)
{
    const size_t smem = sizeof(PassSmem<KeyT, kHasVal>);
    // The shared-memory limit above 48 KB is an attribute of the function in each CUDA context (the
    // module is loaded per context), so it is set before every launch: a flag per device or per
    // context handle would miss a context created after the first call, or one re-created at the
    // same address.  Setting it again is a cheap host call and changes nothing.
    cudaError_t e = cudaFuncSetAttribute(k_pass<KeyT, kHasVal>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_pass<KeyT, kHasVal><<<num_tiles(n), kThreads, smem, s>>>(kin, kout, vin, vout, n, bit, pass, h, lookback);
    return cudaGetLastError();
}

template <class KeyT>
cudaError_t launch_passes(KeyT* keys, uint32_t* vals, KeyT* tmpKeys, uint32_t* tmpVals, uint32_t n, int startBit,
                          int nPasses, Header* h, unsigned long long* lookback, cudaStream_t s)
{
    KeyT* src = keys;
    KeyT* dst = tmpKeys;
    uint32_t* vsrc = vals;
    uint32_t* vdst = tmpVals;
    for (int p = 0; p < nPasses; p++) {
        cudaError_t e = vals ? launch_pass<KeyT, true>(src, dst, vsrc, vdst, n, startBit + 8 * p, p, h, lookback, s)
                             : launch_pass<KeyT, false>(src, dst, nullptr, nullptr, n, startBit + 8 * p, p, h,
                                                        lookback, s);
        if (e != cudaSuccess) return e;
        KeyT* t = src; src = dst; dst = t;
        uint32_t* tv = vsrc; vsrc = vdst; vdst = tv;
    }
    if (src != keys) {  // odd number of passes: result is in tmp (tinyhiponesweep.h:659-667)
        cudaError_t e = cudaMemcpyAsync(keys, src, sizeof(KeyT) * (size_t)n, cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess) return e;
        if (vals) e = cudaMemcpyAsync(vals, vsrc, sizeof(uint32_t) * (size_t)n, cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

template cudaError_t launch_hist<uint32_t>(const uint32_t*, uint32_t, int, int, Header*, unsigned long long*, cudaStream_t);
template cudaError_t launch_hist<unsigned long long>(const unsigned long long*, uint32_t, int, int, Header*,
                                                     unsigned long long*, cudaStream_t);
template cudaError_t launch_passes<uint32_t>(uint32_t*, uint32_t*, uint32_t*, uint32_t*, uint32_t, int, int, Header*,
                                             unsigned long long*, cudaStream_t);
template cudaError_t launch_passes<unsigned long long>(unsigned long long*, uint32_t*, unsigned long long*, uint32_t*,
                                                       uint32_t, int, int, Header*, unsigned long long*, cudaStream_t);

}  // namespace sort
}  // namespace pz
