// sort.cu -- stable LSD radix sort of (Morton key, index) pairs and the
// permutation gathers (src/core/state.py:20-40: cp.argsort + 8 gathers).
//
// cnb_sort_pairs, one sweep per 8-bit digit:
//   k_digit_hist_all  the counts of every digit of every pass, one read of
//                     the keys (runs of equal digits summed in registers)
//   k_onesweep        per 2048-key tile (tiles handed out in order by an
//                     atomic counter): stable in-tile ranks (warp
//                     __match_any_sync + per-warp digit counters), the tile's
//                     digit counts published at once, the counts of earlier
//                     tiles gathered by looking back at what they published
//                     (bounded waits on tiles that already started), the tile
//                     reordered by digit in shared memory and written out in
//                     coalesced runs
// One pass reads 12 B and writes 12 B per key.  Tiles are 2048 keys.
//
// cnb_sort_pairs_noalloc keeps the reduce-then-scan form, which never waits
// on another block: per pass k_digit_count (per-tile counts), k_scan_rows
// (one block per digit) and k_scatter.
#include <new>

#include "ctx.cuh"

namespace cnb {

__global__ void __launch_bounds__(kSortThreads) k_digit_count(const uint64_t *__restrict__ keys,
                                                              int64_t n, int shift,
                                                              uint32_t *__restrict__ hist,
                                                              int64_t tiles) {
    __shared__ uint32_t wh[kSortThreads / 32][256];
    const int warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < (kSortThreads / 32) * 256; i += kSortThreads) (&wh[0][0])[i] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kSortTile;
#pragma unroll 4
    for (int r = 0; r < kSortItems; ++r) {
        int64_t e = base + (int64_t)r * kSortThreads + threadIdx.x;
        if (e < n) {
            uint32_t d = (uint32_t)(__ldg(keys + e) >> shift) & 255u;
            atomicAdd(&wh[warp][d], 1u);
        }
    }
    __syncthreads();
    for (int d = threadIdx.x; d < 256; d += kSortThreads) {
        uint32_t s = 0;
#pragma unroll
        for (int w = 0; w < kSortThreads / 32; ++w) s += wh[w][d];
        hist[(int64_t)d * tiles + blockIdx.x] = s;
    }
}

// Exclusive scan of one digit's row of tile counts (in place), one block per
// digit; the row total goes to totals[digit].
__global__ void __launch_bounds__(256) k_scan_rows(uint32_t *__restrict__ hist, int64_t tiles,
                                                   uint32_t *__restrict__ totals) {
    __shared__ uint32_t warp_sums[8];
    __shared__ uint32_t carry;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t *row = hist + (int64_t)blockIdx.x * tiles;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int64_t base = 0; base < tiles; base += 256 * 4) {
        uint32_t v[4];
        uint32_t local = 0;
        const int64_t b0 = base + (int64_t)threadIdx.x * 4;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            v[k] = (b0 + k < tiles) ? row[b0 + k] : 0u;
            local += v[k];
        }
        uint32_t incl = local;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        if (lane == 31) warp_sums[warp] = incl;
        __syncthreads();
        uint32_t wbase = 0, total = 0;
#pragma unroll
        for (int w = 0; w < 8; ++w) {
            wbase += (w < warp) ? warp_sums[w] : 0u;
            total += warp_sums[w];
        }
        uint32_t run = carry + wbase + (incl - local);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (b0 + k < tiles) row[b0 + k] = run;
            run += v[k];
        }
        __syncthreads();
        if (threadIdx.x == 0) carry += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) totals[blockIdx.x] = carry;
}

// Exclusive block scan of 256 values held one per thread (blockDim == 256).
__device__ __forceinline__ uint32_t block_exscan256(uint32_t v, uint32_t *warp_sums) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) warp_sums[warp] = incl;
    __syncthreads();
    uint32_t wbase = 0;
#pragma unroll
    for (int w = 0; w < 8; ++w) wbase += (w < warp) ? warp_sums[w] : 0u;
    __syncthreads();
    return wbase + incl - v;
}

constexpr int kScatterSmem = kSortTile * (sizeof(uint64_t) + sizeof(uint32_t));

// One pass of the LSD sort over a 4096-key tile: stable ranks within the
// tile (warp __match_any_sync + per-warp digit counters), the tile sorted by
// digit in shared memory, then written out in runs so that consecutive
// threads store consecutive global positions.
template <bool IDENTITY_IN>
__global__ void __launch_bounds__(kSortThreads) k_scatter(const uint64_t *__restrict__ kin,
                                                          const uint32_t *__restrict__ vin,
                                                          uint64_t *__restrict__ kout,
                                                          uint32_t *__restrict__ vout,
                                                          int64_t n, int shift,
                                                          const uint32_t *__restrict__ offs,
                                                          const uint32_t *__restrict__ totals,
                                                          int64_t tiles) {
    static_assert(kSortThreads == 256, "block scans assume 256 threads");
    constexpr int W = kSortThreads / 32;
    extern __shared__ __align__(16) unsigned char smem[];
    uint64_t *skey = reinterpret_cast<uint64_t *>(smem);
    uint32_t *sval = reinterpret_cast<uint32_t *>(smem + kSortTile * sizeof(uint64_t));
    __shared__ uint32_t wcnt[W][257];
    __shared__ uint32_t gbase[256];
    __shared__ uint32_t tstart[256];
    __shared__ uint32_t wsum[8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < W * 257; i += kSortThreads) (&wcnt[0][0])[i] = 0;
    {
        // global start of each digit: digits before it + this digit in earlier tiles
        const int d = threadIdx.x;
        const uint32_t base = block_exscan256(totals[d], wsum);
        gbase[d] = base + offs[(int64_t)d * tiles + blockIdx.x];
    }
    __syncthreads();

    const uint32_t lt_mask = (1u << lane) - 1u;
    const int64_t tbase = (int64_t)blockIdx.x * kSortTile;
    const int64_t wbase = tbase + (int64_t)warp * 32 * kSortItems;
    uint64_t key[kSortItems];
    uint32_t val[kSortItems];
    uint32_t rank[kSortItems];
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        const int64_t e = wbase + r * 32 + lane;
        uint32_t d = 256;  // sentinel for lanes past the end
        if (e < n) {
            key[r] = kin[e];
            val[r] = IDENTITY_IN ? (uint32_t)e : vin[e];
            d = (uint32_t)(key[r] >> shift) & 255u;
        } else {
            key[r] = 0;
            val[r] = 0;
        }
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        const uint32_t before = wcnt[warp][d];
        __syncwarp();
        if ((peers & lt_mask) == 0) wcnt[warp][d] = before + __popc(peers);
        __syncwarp();
        rank[r] = before + __popc(peers & lt_mask);
    }
    __syncthreads();
    {
        // per digit: exclusive prefix over warps, then the digit's start in the tile
        const int d = threadIdx.x;
        uint32_t run = 0;
#pragma unroll
        for (int w = 0; w < W; ++w) {
            const uint32_t c = wcnt[w][d];
            wcnt[w][d] = run;
            run += c;
        }
        tstart[d] = block_exscan256(run, wsum);
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        const int64_t e = wbase + r * 32 + lane;
        if (e < n) {
            const uint32_t d = (uint32_t)(key[r] >> shift) & 255u;
            const uint32_t lp = tstart[d] + wcnt[warp][d] + rank[r];
            skey[lp] = key[r];
            sval[lp] = val[r];
        }
    }
    __syncthreads();
    const int tile_n = (int)min((int64_t)kSortTile, n - tbase);
    for (int j = threadIdx.x; j < tile_n; j += kSortThreads) {
        const uint64_t k = skey[j];
        const uint32_t d = (uint32_t)(k >> shift) & 255u;
        const int64_t pos = (int64_t)gbase[d] + (j - tstart[d]);
        kout[pos] = k;
        vout[pos] = sval[j];
    }
}

// ---------------------------------------------------------------- one sweep
// Counts of every digit of the first `passes` passes.  Each thread sums
// runs of equal digits over kSortItems consecutive keys before touching the
// shared histograms (sorted or nearly sorted input repeats its high digits).
// skip: a device flag set when the near-sorted path already produced the
// result (every kernel of the full sort then returns at once); runs: counts
// the full sorts that ran.
__global__ void __launch_bounds__(kSortThreads) k_digit_hist_all(const uint64_t *__restrict__ keys,
                                                                 int64_t n, int passes,
                                                                 uint32_t *__restrict__ hist,
                                                                 const int32_t *skip,
                                                                 unsigned long long *runs) {
    __shared__ uint32_t sh[kSweepPasses][256];
    if (skip && *(volatile const int32_t *)skip) return;
    if (runs && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(runs, 1ull);
    for (int i = threadIdx.x; i < kSweepPasses * 256; i += kSortThreads) (&sh[0][0])[i] = 0;
    __syncthreads();
    for (int64_t base = ((int64_t)blockIdx.x * kSortThreads + threadIdx.x) * kSortItems; base < n;
         base += (int64_t)gridDim.x * kSortThreads * kSortItems) {
        const int cnt = (int)min((int64_t)kSortItems, n - base);
        uint64_t kk[kSortItems];
#pragma unroll
        for (int k = 0; k < kSortItems; ++k) kk[k] = (k < cnt) ? __ldg(keys + base + k) : 0;
        for (int p = 0; p < passes; ++p) {
            const int shift = 8 * p;
            uint32_t cur = (uint32_t)(kk[0] >> shift) & 255u, run = 1;
#pragma unroll
            for (int k = 1; k < kSortItems; ++k) {
                if (k < cnt) {
                    const uint32_t d = (uint32_t)(kk[k] >> shift) & 255u;
                    if (d == cur) {
                        ++run;
                    } else {
                        atomicAdd(&sh[p][cur], run);
                        cur = d;
                        run = 1;
                    }
                }
            }
            atomicAdd(&sh[p][cur], run);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < passes * 256; i += kSortThreads) {
        const uint32_t v = (&sh[0][0])[i];
        if (v) atomicAdd(hist + i, v);
    }
}

// Look-back words: the tile's count of one digit in the low 32 bits, the
// state above (0: not yet published, 1: this tile's count only, 2: the
// count of this and every earlier tile).
constexpr uint64_t kLbCount = 1ull << 32, kLbPrefix = 2ull << 32;
// the one-sweep tile and how many earlier tiles one look-back step reads
constexpr int kSweepThreads = 512;  // 16 warps: a short ranking chain, 32 warps per SM
constexpr int kSweepItems = 8;
constexpr int kLookbackWindow = 4;
constexpr int kSweepTile = kSweepThreads * kSweepItems;
constexpr int kSweepSmem = kSweepTile * (sizeof(uint64_t) + sizeof(uint32_t));
static_assert(kSweepTile >= 2048, "sweep_bytes() sizes the look-back words for 2048-key tiles");
constexpr int kLookbackSpinLimit = 1 << 22;

__device__ __forceinline__ void lb_store(uint64_t *p, uint64_t v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ uint64_t lb_load(const uint64_t *p) {
    uint64_t v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// Exclusive scan over the NT threads of a block (one value each).
template <int NT>
__device__ __forceinline__ uint32_t block_exscan(uint32_t v, uint32_t *warp_sums) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) warp_sums[warp] = incl;
    __syncthreads();
    uint32_t wbase = 0;
#pragma unroll
    for (int w = 0; w < NT / 32; ++w) wbase += (w < warp) ? warp_sums[w] : 0u;
    __syncthreads();
    return wbase + incl - v;
}

template <bool IDENTITY_IN>
__global__ void __launch_bounds__(kSweepThreads) k_onesweep(const uint64_t *__restrict__ kin,
                                                           const uint32_t *__restrict__ vin,
                                                           uint64_t *__restrict__ kout,
                                                           uint32_t *__restrict__ vout,
                                                           int64_t n, int shift,
                                                           const uint32_t *__restrict__ hist,
                                                           uint64_t *lookback,
                                                           int32_t *tile_counter,
                                                           int32_t *flags, const int32_t *skip,
                                                           int wait_limit, int64_t withheld) {
    static_assert(kSweepThreads >= 256, "one thread per digit");
    if (skip && *(volatile const int32_t *)skip) return;
    constexpr int W = kSweepThreads / 32;
    extern __shared__ __align__(16) unsigned char smem[];
    uint64_t *skey = reinterpret_cast<uint64_t *>(smem);
    uint32_t *sval = reinterpret_cast<uint32_t *>(smem + kSweepTile * sizeof(uint64_t));
    __shared__ uint32_t wcnt[W][257];
    __shared__ uint32_t gbase[256];
    __shared__ uint32_t tstart[256];
    __shared__ uint32_t wsum[W];
    __shared__ int s_tile;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const bool digit_thread = threadIdx.x < 256;
    // tiles in the order blocks start: every tile this one waits for has started
    if (threadIdx.x == 0) s_tile = atomicAdd(tile_counter, 1);
    for (int i = threadIdx.x; i < W * 257; i += kSweepThreads) (&wcnt[0][0])[i] = 0;
    // start of each digit among all keys (threads 0..255, one digit each)
    const uint32_t digit_start = block_exscan<kSweepThreads>(digit_thread ? hist[threadIdx.x] : 0u, wsum);
    __syncthreads();
    const int64_t tile = s_tile;

    const uint32_t lt_mask = (1u << lane) - 1u;
    const int64_t tbase = tile * kSweepTile;
    const int64_t wbase = tbase + (int64_t)warp * 32 * kSweepItems;
    uint64_t key[kSweepItems];
    uint32_t val[kSweepItems];
    uint32_t rank[kSweepItems];
    // every load of the tile in flight before the first is used
#pragma unroll
    for (int r = 0; r < kSweepItems; ++r) {
        const int64_t e = wbase + r * 32 + lane;
        key[r] = e < n ? __ldcs(kin + e) : 0;
        val[r] = IDENTITY_IN ? (uint32_t)e : (e < n ? __ldcs(vin + e) : 0u);
    }
#pragma unroll
    for (int r = 0; r < kSweepItems; ++r) {
        const int64_t e = wbase + r * 32 + lane;
        // sentinel digit 256 for lanes past the end
        const uint32_t d = e < n ? (uint32_t)(key[r] >> shift) & 255u : 256u;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        const uint32_t before = wcnt[warp][d];
        __syncwarp();
        if ((peers & lt_mask) == 0) wcnt[warp][d] = before + __popc(peers);
        __syncwarp();
        rank[r] = before + __popc(peers & lt_mask);
    }
    __syncthreads();
    {
        const int d = threadIdx.x;
        uint32_t run = 0;
        uint32_t before = 0;
        if (digit_thread) {
#pragma unroll
            for (int w = 0; w < W; ++w) {
                const uint32_t c = wcnt[w][d];
                wcnt[w][d] = run;
                run += c;
            }
            // publish this tile's count, then add up the earlier tiles' counts
            uint64_t *mine = lookback + tile * 256 + d;
            // a withheld tile (cnb_ctx_inject_sort_faults) keeps its counts to
            // itself: the tiles after it wait until their limit
            const bool publish = tile != withheld;
            if (tile == 0) {
                if (publish) lb_store(mine, kLbPrefix | run);
            } else {
                if (publish) lb_store(mine, kLbCount | run);
                // kLookbackWindow earlier tiles per round trip, used in order up
                // to the first one not yet published (tile 0 always ends the walk)
                int64_t j = tile - 1;
                int spins = 0;
                for (;;) {
                    uint64_t v[kLookbackWindow];
#pragma unroll
                    for (int w = 0; w < kLookbackWindow; ++w)
                        v[w] = (j - w >= 0) ? lb_load(lookback + (j - w) * 256 + d) : kLbPrefix;
                    int used = 0;
                    bool done = false;
#pragma unroll
                    for (int w = 0; w < kLookbackWindow; ++w) {
                        const uint32_t state = (uint32_t)(v[w] >> 32);
                        if (!done && used == w && state != 0) {
                            before += (uint32_t)v[w];
                            used = w + 1;
                            done = (state == 2);
                        }
                    }
                    if (done) break;
                    j -= used;
                    if (used == 0) {
                        if (++spins > wait_limit) {
                            set_flag(flags, CNB_FLAG_WAIT_LIMIT);
                            break;
                        }
                        if (spins > 16) __nanosleep(64);
                    }
                }
                if (publish) lb_store(mine, kLbPrefix | (before + run));
            }
            gbase[d] = digit_start + before;
        }
        const uint32_t ts = block_exscan<kSweepThreads>(run, wsum);
        if (digit_thread) tstart[d] = ts;
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kSweepItems; ++r) {
        const int64_t e = wbase + r * 32 + lane;
        if (e < n) {
            const uint32_t d = (uint32_t)(key[r] >> shift) & 255u;
            const uint32_t lp = tstart[d] + wcnt[warp][d] + rank[r];
            skey[lp] = key[r];
            sval[lp] = val[r];
        }
    }
    __syncthreads();
    const int tile_n = (int)min((int64_t)kSweepTile, n - tbase);
    for (int j = threadIdx.x; j < tile_n; j += kSweepThreads) {
        const uint64_t k = skey[j];
        const uint32_t d = (uint32_t)(k >> shift) & 255u;
        const int64_t pos = (int64_t)gbase[d] + (j - tstart[d]);
        kout[pos] = k;
        vout[pos] = sval[j];
    }
}

__global__ void __launch_bounds__(256) k_zero_words(uint64_t *p, int64_t words,
                                                    const int32_t *skip) {
    if (*(volatile const int32_t *)skip) return;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < words;
         i += (int64_t)gridDim.x * blockDim.x)
        p[i] = 0ull;
}

__global__ void k_take_flags(int32_t *ctx_flags, int32_t *status) {
    const int32_t f = *ctx_flags;
    if (f) {
        atomicOr(status, f);
        *ctx_flags = 0;
    }
}

int sort_pairs_onesweep(cnb_ctx *ctx, const uint64_t *keys_in, uint64_t *keys_out,
                        const uint32_t *idx_in, uint32_t *perm_out, int64_t n, int key_bits,
                        cudaStream_t st, const int32_t *skip) {
    if (n == 0) return CNB_OK;
    int passes = (key_bits + 7) / 8;
    if (passes < 1) passes = 1;
    if (passes == 1 && (keys_in == keys_out || (idx_in && idx_in == perm_out))) passes = 2;
    const int64_t tiles = (n + kSweepTile - 1) / kSweepTile;
    uint32_t *hist = ctx->sweep;
    int32_t *counters = reinterpret_cast<int32_t *>(ctx->sweep + kSweepPasses * 256);
    uint64_t *lookback = reinterpret_cast<uint64_t *>(ctx->sweep + kSweepMetaWords);
    const size_t zero_bytes = kSweepMetaWords * 4 + (size_t)passes * tiles * 256 * 8;
    if (skip) {
        // zeroed on the device only when this sort runs
        static_assert((kSweepMetaWords * 4) % 8 == 0, "whole 64-bit words");
        const int64_t words = (int64_t)(zero_bytes / 8);
        k_zero_words<<<grid_for(words, 256, 148 * 8), 256, 0, st>>>(
            reinterpret_cast<uint64_t *>(ctx->sweep), words, skip);
        CNB_TRY(launch_status());
    } else {
        CNB_CUDA(cudaMemsetAsync(ctx->sweep, 0, zero_bytes, st));
    }
    CNB_CUDA(cudaFuncSetAttribute(k_onesweep<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  kSweepSmem));
    CNB_CUDA(cudaFuncSetAttribute(k_onesweep<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  kSweepSmem));
    k_digit_hist_all<<<grid_for(n, kSortTile, 148 * 8), kSortThreads, 0, st>>>(
        keys_in, n, passes, hist, skip, ctx->sort_stats ? ctx->sort_stats + 1 : nullptr);
    CNB_TRY(launch_status());
    const uint64_t *ks = keys_in;
    const uint32_t *vs = idx_in;
    const int wait_limit = ctx->wait_limit > 0 ? ctx->wait_limit : kLookbackSpinLimit;
    for (int p = 0; p < passes; ++p) {
        const bool last = (p == passes - 1);
        uint64_t *kd = last ? keys_out : ctx->keys_tmp[p & 1];
        uint32_t *vd = last ? perm_out : ctx->vals_tmp[p & 1];
        uint64_t *lb = lookback + (int64_t)p * tiles * 256;
        if (vs == nullptr)
            k_onesweep<true><<<(unsigned)tiles, kSweepThreads, kSweepSmem, st>>>(
                ks, nullptr, kd, vd, n, 8 * p, hist + 256 * p, lb, counters + p, ctx->flags, skip,
                wait_limit, ctx->withheld_tile);
        else
            k_onesweep<false><<<(unsigned)tiles, kSweepThreads, kSweepSmem, st>>>(
                ks, vs, kd, vd, n, 8 * p, hist + 256 * p, lb, counters + p, ctx->flags, skip,
                wait_limit, ctx->withheld_tile);
        CNB_TRY(launch_status());
        ks = kd;
        vs = vd;
    }
    return CNB_OK;
}

struct GatherArgs {
    const float *src[8];
    float *dst[8];
};

template <int K>
__global__ void __launch_bounds__(256) k_gather_f32(const uint32_t *__restrict__ perm,
                                                    GatherArgs a, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        uint32_t p = __ldcs(perm + i);
#pragma unroll
        for (int k = 0; k < K; ++k) a.dst[k][i] = __ldg(a.src[k] + p);
    }
}

int sort_pairs(cnb_ctx *ctx, const uint64_t *keys_in, uint64_t *keys_out,
               const uint32_t *idx_in, uint32_t *perm_out, int64_t n, int key_bits,
               cudaStream_t st) {
    if (n == 0) return CNB_OK;
    int passes = (key_bits + 7) / 8;
    if (passes < 1) passes = 1;
    if (passes == 1 && (keys_in == keys_out || (idx_in && idx_in == perm_out))) passes = 2;
    const int64_t tiles = (n + kSortTile - 1) / kSortTile;
    // the scatter's staging tile is above the 48 KB default (cheap host call)
    CNB_CUDA(cudaFuncSetAttribute(k_scatter<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  kScatterSmem));
    CNB_CUDA(cudaFuncSetAttribute(k_scatter<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  kScatterSmem));
    const uint64_t *ks = keys_in;
    const uint32_t *vs = idx_in;
    for (int p = 0; p < passes; ++p) {
        const int shift = 8 * p;
        const bool last = (p == passes - 1);
        uint64_t *kd = last ? keys_out : ctx->keys_tmp[p & 1];
        uint32_t *vd = last ? perm_out : ctx->vals_tmp[p & 1];
        uint32_t *totals = ctx->tile_hist + 256 * tiles;
        k_digit_count<<<(unsigned)tiles, kSortThreads, 0, st>>>(ks, n, shift, ctx->tile_hist,
                                                               tiles);
        CNB_TRY(launch_status());
        k_scan_rows<<<256, 256, 0, st>>>(ctx->tile_hist, tiles, totals);
        CNB_TRY(launch_status());
        if (vs == nullptr)
            k_scatter<true><<<(unsigned)tiles, kSortThreads, kScatterSmem, st>>>(
                ks, nullptr, kd, vd, n, shift, ctx->tile_hist, totals, tiles);
        else
            k_scatter<false><<<(unsigned)tiles, kSortThreads, kScatterSmem, st>>>(
                ks, vs, kd, vd, n, shift, ctx->tile_hist, totals, tiles);
        CNB_TRY(launch_status());
        ks = kd;
        vs = vd;
    }
    return CNB_OK;
}

int gather_f32(const uint32_t *perm, int n_arrays, const float *const *src, float *const *dst,
               int64_t n, cudaStream_t st) {
    GatherArgs a{};
    for (int k = 0; k < n_arrays; ++k) {
        a.src[k] = src[k];
        a.dst[k] = dst[k];
    }
    const int g = grid_for(n, 256, 148 * 16);
    switch (n_arrays) {
#define CNB_G(K) \
    case K: k_gather_f32<K><<<g, 256, 0, st>>>(perm, a, n); break;
        CNB_G(1) CNB_G(2) CNB_G(3) CNB_G(4) CNB_G(5) CNB_G(6) CNB_G(7) CNB_G(8)
#undef CNB_G
        default: return CNB_E_INVALID_ARG;
    }
    return launch_status();
}

}  // namespace cnb

extern "C" int cnb_ctx_create(int64_t n_max, cnb_ctx **out) {
    if (!out || n_max < 0) return CNB_E_INVALID_ARG;
    if (n_max > (int64_t)UINT32_MAX) return CNB_E_TOO_LARGE;
    *out = nullptr;
    cnb_ctx *c = new (std::nothrow) cnb_ctx();
    if (!c) return CNB_E_NO_MEMORY;
    cudaGetDevice(&c->device);
    c->n_max = n_max;
    int64_t nn = n_max > 0 ? n_max : 1;
    c->tiles_max = (nn + cnb::kSortTile - 1) / cnb::kSortTile;
    cudaError_t e = cudaSuccess;
    for (int k = 0; k < 2 && e == cudaSuccess; ++k) {
        e = cudaMalloc(&c->keys_tmp[k], sizeof(uint64_t) * nn);
        if (e == cudaSuccess) e = cudaMalloc(&c->vals_tmp[k], sizeof(uint32_t) * nn);
    }
    if (e == cudaSuccess) e = cudaMalloc(&c->sweep, cnb::sweep_bytes(nn));
    if (e == cudaSuccess) e = cudaMalloc(&c->flags, sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMemset(c->flags, 0, sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMalloc(&c->near, cnb::near_bytes(nn));
    if (e == cudaSuccess) e = cudaMalloc(&c->sort_stats, 2 * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemset(c->sort_stats, 0, 2 * sizeof(unsigned long long));
    if (e != cudaSuccess) {
        cnb_ctx_destroy(c);
        cnb::record_cuda_error(e);
        return CNB_E_NO_MEMORY;
    }
    *out = c;
    return CNB_OK;
}

extern "C" int cnb_ctx_destroy(cnb_ctx *c) {
    if (!c) return CNB_OK;
    for (int k = 0; k < 2; ++k) {
        cudaFree(c->keys_tmp[k]);
        cudaFree(c->vals_tmp[k]);
    }
    cudaFree(c->tile_hist);
    cudaFree(c->sweep);
    cudaFree(c->flags);
    cudaFree(c->near);
    cudaFree(c->sort_stats);
    if (c->side) cudaStreamDestroy(c->side);
    cudaFree(c->group_scratch);
    delete c;
    return CNB_OK;
}

extern "C" int cnb_sort_pairs(cnb_ctx *ctx, const uint64_t *keys_in, uint64_t *keys_out,
                              const uint32_t *idx_in, uint32_t *perm_out, int64_t n,
                              int key_bits, void *stream) {
    if (!ctx || n < 0 || key_bits < 1 || key_bits > 64) return CNB_E_INVALID_ARG;
    if (n > ctx->n_max) return CNB_E_TOO_LARGE;
    if (n > 0 && (!keys_in || !keys_out || !perm_out)) return CNB_E_INVALID_ARG;
    if (!cnb::sort_buffers_ok(keys_in, keys_out, idx_in, perm_out, n)) return CNB_E_INVALID_ARG;
    cudaStream_t st = cnb::as_stream(stream);
    const int32_t *skip = nullptr, *never = nullptr;
    if (!(ctx->sort_mode == CNB_SORT_ADAPTIVE && n > 0 && idx_in == nullptr && keys_in != keys_out))
        return cnb::sort_pairs_onesweep(ctx, keys_in, keys_out, idx_in, perm_out, n, key_bits, st);
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CNB_CUDA(cudaStreamIsCapturing(st, &cs));
    if (cs != cudaStreamCaptureStatusActive) {
        // eager: the full sort's kernels follow and return at once when the
        // near-sorted path produced the result
        CNB_TRY(cnb::sort_pairs_near(ctx, keys_in, keys_out, perm_out, n, st, &skip, &never, 0,
                                     false));
        return cnb::sort_pairs_onesweep(ctx, keys_in, keys_out, nullptr, perm_out, n, key_bits,
                                        st, skip);
    }
    // captured: the full sort goes into the body of a conditional node that
    // runs unless the near-sorted path clears it (default 1 at every launch)
    cudaGraph_t g = nullptr;
    CNB_CUDA(cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, nullptr, nullptr));
    cudaGraphConditionalHandle cond;
    CNB_CUDA(cudaGraphConditionalHandleCreate(&cond, g, 1u, cudaGraphCondAssignDefault));
    CNB_TRY(cnb::sort_pairs_near(ctx, keys_in, keys_out, perm_out, n, st, &skip, &never, cond,
                                 true));
    const cudaGraphNode_t *deps = nullptr;
    size_t nd = 0;
    CNB_CUDA(cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &nd));
    cudaGraphNodeParams p = {};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = cond;
    p.conditional.type = cudaGraphCondTypeIf;
    p.conditional.size = 1;
    cudaGraphNode_t node;
    CNB_CUDA(cudaGraphAddNode(&node, g, deps, nd, &p));
    cudaGraph_t body = p.conditional.phGraph_out[0];
    if (!ctx->side) CNB_CUDA(cudaStreamCreateWithFlags(&ctx->side, cudaStreamNonBlocking));
    CNB_CUDA(cudaStreamBeginCaptureToGraph(ctx->side, body, nullptr, nullptr, 0,
                                           cudaStreamCaptureModeRelaxed));
    // `never` keeps the body's zeroing a kernel (the flag it reads stays 0)
    const int rc = cnb::sort_pairs_onesweep(ctx, keys_in, keys_out, nullptr, perm_out, n, key_bits,
                                            ctx->side, never);
    cudaGraph_t captured = nullptr;
    const cudaError_t e = cudaStreamEndCapture(ctx->side, &captured);
    CNB_TRY(rc);
    CNB_CUDA(e);
    CNB_CUDA(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies));
    return CNB_OK;
}

extern "C" int cnb_ctx_set_sort_mode(cnb_ctx *ctx, int mode) {
    if (!ctx || (mode != CNB_SORT_FULL && mode != CNB_SORT_ADAPTIVE)) return CNB_E_INVALID_ARG;
    ctx->sort_mode = mode;
    return CNB_OK;
}

extern "C" int cnb_ctx_inject_sort_faults(cnb_ctx *ctx, int32_t wait_limit,
                                          int64_t withheld_tile, int64_t near_dest_bias) {
    if (!ctx || wait_limit < 0 || withheld_tile < -1 || near_dest_bias < 0)
        return CNB_E_INVALID_ARG;
    ctx->wait_limit = wait_limit;
    ctx->withheld_tile = withheld_tile;
    ctx->near_dest_bias = near_dest_bias;
    return CNB_OK;
}

extern "C" int cnb_ctx_sort_stats(cnb_ctx *ctx, int64_t *out) {
    if (!ctx || !out) return CNB_E_INVALID_ARG;
    unsigned long long v[2];
    CNB_CUDA(cudaDeviceSynchronize());
    CNB_CUDA(cudaMemcpy(v, ctx->sort_stats, sizeof(v), cudaMemcpyDeviceToHost));
    out[0] = (int64_t)v[0];
    out[1] = (int64_t)v[1];
    return CNB_OK;
}

extern "C" int cnb_ctx_take_flags(cnb_ctx *ctx, int32_t *status, void *stream) {
    if (!ctx || !status) return CNB_E_INVALID_ARG;
    cnb::k_take_flags<<<1, 1, 0, cnb::as_stream(stream)>>>(ctx->flags, status);
    return cnb::launch_status();
}

extern "C" int cnb_gather_f32(const uint32_t *perm, int n_arrays, const float *const *src,
                              float *const *dst, int64_t n, void *stream) {
    if (n < 0 || n_arrays < 1 || n_arrays > 8 || !src || !dst) return CNB_E_INVALID_ARG;
    if (n == 0) return CNB_OK;
    if (!perm) return CNB_E_INVALID_ARG;
    for (int k = 0; k < n_arrays; ++k)
        if (!src[k] || !dst[k] || src[k] == dst[k]) return CNB_E_INVALID_ARG;
    return cnb::gather_f32(perm, n_arrays, src, dst, n, cnb::as_stream(stream));
}
