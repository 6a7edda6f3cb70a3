// sort_near.cu -- the near-sorted path of the adaptive sort
// (CNB_SORT_ADAPTIVE; src/core/state.py:35 `cp.argsort(codes)` on keys that
// were sorted one step earlier).
//
// Between two steps a body keeps its place in the Morton order unless it
// crossed the periodic boundary or overtook a neighbour, so the keys ascend
// except in a few places.  The path takes out a set S of keys such that the
// rest R ascends, sorts S, and merges S back into R.  The result is exactly
// the stable argsort (ties by index), the same as the full radix sort's.
// Four kernels over 4096-key tiles; the last block of each of the first three
// to finish (a completion counter, no waiting) does the step that needs every
// tile's result:
//   k_near_mark    a tile whose keys ascend, together with the key before and
//                  the key after it, is clean (one coalesced read).  In the
//                  others, over the tile and 128 keys either side: at every
//                  descent a > b among the unmarked keys, mark the run after
//                  it of keys below a or the run before it of keys above b,
//                  whichever is shorter (a displaced key, or a clump of
//                  neighbours that moved together), until the unmarked keys
//                  ascend.  Per tile the max and min unmarked key.
//                  Last block: per tile the max of the unmarked keys of the
//                  tiles before it and the min of those after it.
//   k_near_filter  S = marked keys, and unmarked keys below the max of the
//                  unmarked keys before them or above the min of those after
//                  them.  R ascends whatever the marking did: for i < j in R,
//                  key(i) <= min(unmarked after i) <= key(j).  Per tile |S| and
//                  the first key of R.  Last block: offsets of S per tile; the
//                  path is taken when |S| <= kNearCap, otherwise the flag it
//                  leaves at 0 lets the full radix sort run (the full sort's
//                  kernels read the flag and return when the path was taken:
//                  the choice needs no host round trip and is captured in a
//                  CUDA graph like any other launch).
//   k_near_take    S in index order.  Last block: S ordered by (key, index) by a
//                  bitonic network in shared memory, and per tile the range of
//                  S keys whose R neighbours fall in the tile.
//   k_near_place   an R key goes to (its rank in R) + (keys of S before it); an
//                  S key goes to (its rank in S) + (keys of R before it), counted
//                  by the tile whose R keys bracket it.  A clean tile with no S
//                  key in its range is a shifted copy.
// Order everywhere is (key, index) lexicographic, so equal keys keep their
// input order.
#include "ctx.cuh"

namespace cnb {

namespace {

constexpr int kNearHalo = 128;                         // keys either side of a tile
constexpr int kNearWin = kNearTile + 2 * kNearHalo;    // 4352
constexpr int kNearWinItems = (kNearWin + kNearThreads - 1) / kNearThreads;
constexpr int kNearMaxDescents = 256;  // more descents in one window: give up
constexpr int kNearRounds = 32;        // marking rounds before giving up
constexpr int kNearReach = 256;        // keys one descent looks at on either side
constexpr int kNearWords = kNearTile / 32;
constexpr size_t kNearMarkSmem = (size_t)kNearWin * (sizeof(uint64_t) + sizeof(uint16_t) + 1);
constexpr size_t kNearPlaceSmem = (size_t)kNearTile * (sizeof(uint64_t) + sizeof(uint32_t));
constexpr uint32_t kNone = 0xffffffffu;
static_assert(kNearWin < 65536, "window positions are 16-bit");
static_assert(kNearItems == 8 && kNearTile % 32 == 0, "eight keys per thread, one byte of a word");

struct NearWs {
    int32_t *ctl;  // [0] give up, [1] near path taken, [2] |S|, [3..5] blocks done per kernel
    uint64_t *umax, *umin, *pmax, *smin, *rkey;  // per tile
    uint32_t *scnt, *soff, *rpos, *dirty, *tlo;  // per tile (soff, tlo: tiles + 1)
    uint32_t *bits;                              // per tile kNearWords words
    uint64_t *s_key, *ss_key;                    // kNearCap
    uint32_t *s_pos, *ss_pos;                    // kNearCap
};

int64_t align16(int64_t b) { return (b + 15) & ~(int64_t)15; }

// carves the workspace for nt tiles; returns the bytes it needs
int64_t near_layout(void *base, int64_t nt, NearWs *w) {
    char *p = static_cast<char *>(base);
    int64_t off = 0;
    auto take = [&](int64_t bytes) {
        char *q = p ? p + off : nullptr;
        off += align16(bytes);
        return q;
    };
    NearWs v{};
    v.ctl = reinterpret_cast<int32_t *>(take(8 * sizeof(int32_t)));
    v.umax = reinterpret_cast<uint64_t *>(take(nt * 8));
    v.umin = reinterpret_cast<uint64_t *>(take(nt * 8));
    v.pmax = reinterpret_cast<uint64_t *>(take(nt * 8));
    v.smin = reinterpret_cast<uint64_t *>(take(nt * 8));
    v.rkey = reinterpret_cast<uint64_t *>(take(nt * 8));
    v.scnt = reinterpret_cast<uint32_t *>(take(nt * 4));
    v.soff = reinterpret_cast<uint32_t *>(take((nt + 1) * 4));
    v.rpos = reinterpret_cast<uint32_t *>(take(nt * 4));
    v.dirty = reinterpret_cast<uint32_t *>(take(nt * 4));
    v.tlo = reinterpret_cast<uint32_t *>(take((nt + 1) * 4));
    v.bits = reinterpret_cast<uint32_t *>(take(nt * kNearWords * 4));
    v.s_key = reinterpret_cast<uint64_t *>(take(kNearCap * 8));
    v.ss_key = reinterpret_cast<uint64_t *>(take(kNearCap * 8));
    v.s_pos = reinterpret_cast<uint32_t *>(take(kNearCap * 4));
    v.ss_pos = reinterpret_cast<uint32_t *>(take(kNearCap * 4));
    if (w) *w = v;
    return off;
}

__device__ __forceinline__ bool pair_less(uint64_t ka, uint32_t pa, uint64_t kb, uint32_t pb) {
    return ka < kb || (ka == kb && pa < pb);
}

// Exclusive sum over the block's threads (one value each).
template <int NT>
__device__ __forceinline__ uint32_t near_exsum(uint32_t v, uint32_t *wsum) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    uint32_t base = 0;
    for (int w = 0; w < warp; ++w) base += wsum[w];
    __syncthreads();
    return base + incl - v;
}

// Exclusive max (FWD: over lower thread indices) or min (!FWD: over higher
// thread indices) of 64-bit values across the block.
template <int NT, bool FWD>
__device__ __forceinline__ uint64_t near_exscan64(uint64_t v, uint64_t *wtot) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int W = NT / 32;
    const uint64_t ident = FWD ? 0ull : ~0ull;
    auto op = [](uint64_t a, uint64_t b) { return FWD ? (a > b ? a : b) : (a < b ? a : b); };
    uint64_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint64_t t = FWD ? __shfl_up_sync(0xffffffffu, incl, o)
                               : __shfl_down_sync(0xffffffffu, incl, o);
        if (FWD ? lane >= o : lane + o < 32) incl = op(incl, t);
    }
    if (lane == (FWD ? 31 : 0)) wtot[warp] = incl;
    uint64_t lane_ex = FWD ? __shfl_up_sync(0xffffffffu, incl, 1)
                           : __shfl_down_sync(0xffffffffu, incl, 1);
    if (lane == (FWD ? 0 : 31)) lane_ex = ident;
    __syncthreads();
    uint64_t acc = ident;
    for (int w = 0; w < W; ++w)
        if (FWD ? w < warp : w > warp) acc = op(acc, wtot[w]);
    __syncthreads();
    return op(acc, lane_ex);
}

// the eight bits of this thread's keys in the tile's bit words
__device__ __forceinline__ uint32_t my_byte(const uint32_t *tile_bits) {
    const int j0 = threadIdx.x * kNearItems;
    return (tile_bits[j0 >> 5] >> (j0 & 31)) & 0xffu;
}

// True in every thread of the last block of the grid to get here; the other
// blocks' global writes before their arrival are then visible to it.
__device__ __forceinline__ bool last_block(int32_t *counter, int *s_flag) {
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) *s_flag = (atomicAdd(counter, 1) == (int)gridDim.x - 1);
    __syncthreads();
    const bool last = *s_flag != 0;
    if (last) __threadfence();
    return last;
}

__device__ __forceinline__ int32_t ld_flag(const int32_t *p) { return *(volatile const int32_t *)p; }

// The marking of a tile with a descent (block-uniform control flow).
__device__ void mark_window(const uint64_t *__restrict__ keys, int64_t n, int64_t t, NearWs &w,
                            unsigned char *smem, uint32_t *wsum, int *s_desc, int *s_u,
                            unsigned long long *s_max, unsigned long long *s_min) {
    uint64_t *sk = reinterpret_cast<uint64_t *>(smem);
    uint16_t *ci = reinterpret_cast<uint16_t *>(smem + kNearWin * sizeof(uint64_t));
    uint8_t *mk = smem + kNearWin * (sizeof(uint64_t) + sizeof(uint16_t));
    const int64_t base = t * kNearTile;
    const int64_t lo = base - kNearHalo > 0 ? base - kNearHalo : 0;
    const int64_t hi = base + kNearTile + kNearHalo < n ? base + kNearTile + kNearHalo : n;
    const int wn = (int)(hi - lo);
    const int own0 = (int)(base - lo);
    const int own_n = (int)(n - base < kNearTile ? n - base : kNearTile);
    uint32_t *tile_bits = w.bits + t * kNearWords;
    if (threadIdx.x == 0) {
        *s_desc = 0;
        *s_max = 0ull;
        *s_min = ~0ull;
    }
    {
        uint64_t v[kNearWinItems];
#pragma unroll
        for (int q = 0; q < kNearWinItems; ++q) {
            const int j = threadIdx.x + q * kNearThreads;
            v[q] = j < wn ? __ldg(keys + lo + j) : 0ull;
        }
#pragma unroll
        for (int q = 0; q < kNearWinItems; ++q) {
            const int j = threadIdx.x + q * kNearThreads;
            if (j < wn) {
                sk[j] = v[q];
                mk[j] = 0;
            }
        }
    }
    __syncthreads();
    int desc = 0;
    for (int j = threadIdx.x; j + 1 < wn; j += kNearThreads) desc += sk[j] > sk[j + 1];
    if (desc) atomicAdd(s_desc, desc);
    __syncthreads();
    if (*s_desc > kNearMaxDescents) {
        if (threadIdx.x == 0) atomicExch(w.ctl, 1);
        return;
    }
    bool converged = false;
    for (int r = 0; r < kNearRounds; ++r) {
        // the unmarked window positions in order, a contiguous chunk per thread
        const int c0 = threadIdx.x * kNearWinItems;
        uint32_t cnt = 0;
#pragma unroll
        for (int k = 0; k < kNearWinItems; ++k) {
            const int j = c0 + k;
            cnt += (j < wn && !mk[j]);
        }
        uint32_t off = near_exsum<kNearThreads>(cnt, wsum);
#pragma unroll
        for (int k = 0; k < kNearWinItems; ++k) {
            const int j = c0 + k;
            if (j < wn && !mk[j]) ci[off++] = (uint16_t)j;
        }
        if (threadIdx.x == kNearThreads - 1) *s_u = (int)off;
        __syncthreads();
        const int U = *s_u;
        int changed = 0;
        for (int c = threadIdx.x; c + 1 < U; c += kNearThreads) {
            const uint64_t a = sk[ci[c]], b = sk[ci[c + 1]];
            if (a > b) {
                // the keys after the descent that are below a, and the keys
                // before it that are above b: the shorter side is the one out
                // of place (a displaced key or clump); ties mark the later side.
                // Both runs grow in step until one ends, so the scan stops
                // at the shorter one.
                int kf = 1, kb = 1;
                for (;;) {
                    const bool f = kf < kNearReach && c + 1 + kf < U && sk[ci[c + 1 + kf]] < a;
                    const bool g = kb < kNearReach && c - kb >= 0 && sk[ci[c - kb]] > b;
                    kf += f;
                    kb += g;
                    if (!f || !g) break;
                }
                if (kf <= kb) {
                    for (int q = 1; q <= kf; ++q) mk[ci[c + q]] = 1;
                } else {
                    for (int q = 0; q < kb; ++q) mk[ci[c - q]] = 1;
                }
                changed = 1;
            }
        }
        if (!__syncthreads_or(changed)) {
            converged = true;
            break;
        }
    }
    if (!converged) {
        if (threadIdx.x == 0) atomicExch(w.ctl, 1);
        return;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned long long vmax = 0ull, vmin = ~0ull;
    for (int q = warp; q < kNearWords; q += kNearThreads / 32) {
        const int o = q * 32 + lane;
        const bool own = o < own_n;
        const bool m = own && mk[own0 + o];
        const uint32_t word = __ballot_sync(0xffffffffu, m);
        if (lane == 0) tile_bits[q] = word;
        if (own && !m) {
            const uint64_t k = sk[own0 + o];
            vmax = k > vmax ? k : vmax;
            vmin = k < vmin ? k : vmin;
        }
    }
    if (vmax) atomicMax(s_max, vmax);
    if (vmin != ~0ull) atomicMin(s_min, vmin);
    __syncthreads();
    if (threadIdx.x == 0) {
        w.umax[t] = *s_max;
        w.umin[t] = *s_min;
        w.dirty[t] = 1u;
    }
}

__global__ void __launch_bounds__(kNearThreads) k_near_mark(const uint64_t *__restrict__ keys,
                                                            int64_t n, int64_t nt, NearWs w) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ uint32_t wsum[kNearThreads / 32];
    __shared__ uint64_t wtot[kNearThreads / 32];
    __shared__ int s_desc, s_u, s_last;
    __shared__ unsigned long long s_max, s_min;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t t = blockIdx.x;
    const int64_t base = t * kNearTile;
    const int own_n = (int)(n - base < kNearTile ? n - base : kNearTile);
    // clean test: the tile's keys, the key before it and the key after it
    // ascend (rows of 32 keys per warp, coalesced)
    uint64_t k[kNearItems];
#pragma unroll
    for (int r = 0; r < kNearItems; ++r) {
        const int p = warp * 256 + r * 32 + lane;
        k[r] = p < own_n ? __ldg(keys + base + p) : ~0ull;
    }
    bool desc = false;
#pragma unroll
    for (int r = 0; r < kNearItems; ++r) {
        uint64_t nx = __shfl_down_sync(0xffffffffu, k[r], 1);
        const uint64_t row_next = __shfl_sync(0xffffffffu, k[r < kNearItems - 1 ? r + 1 : r], 0);
        if (lane == 31) {
            if (r < kNearItems - 1) {
                nx = row_next;
            } else {
                const int64_t q = base + warp * 256 + 256;
                nx = q < n ? __ldg(keys + q) : ~0ull;
            }
        }
        const int p = warp * 256 + r * 32 + lane;
        if (p < own_n && k[r] > nx) desc = true;
    }
    if (threadIdx.x == 0 && base > 0 && __ldg(keys + base - 1) > k[0]) desc = true;
    if (!__syncthreads_or(desc)) {
        uint32_t *tile_bits = w.bits + t * kNearWords;
        if (threadIdx.x < kNearWords) tile_bits[threadIdx.x] = 0u;
        if (threadIdx.x == 0) {
            w.umin[t] = k[0];
            w.dirty[t] = 0u;
        }
#pragma unroll
        for (int r = 0; r < kNearItems; ++r)
            if (warp * 256 + r * 32 + lane == own_n - 1) w.umax[t] = k[r];
    } else {
        mark_window(keys, n, t, w, smem, wsum, &s_desc, &s_u, &s_max, &s_min);
    }
    if (!last_block(w.ctl + 3, &s_last) || ld_flag(w.ctl)) return;
    // per tile: max of the unmarked keys of the tiles before, min of those after
    const int64_t per = (nt + kNearThreads - 1) / kNearThreads;
    const int64_t a = (int64_t)threadIdx.x * per;
    const int64_t b = a + per < nt ? a + per : nt;
    uint64_t mx = 0ull, mn = ~0ull;
    for (int64_t i = a; i < b; ++i) {
        const uint64_t u = __ldcg(w.umax + i), v = __ldcg(w.umin + i);
        mx = u > mx ? u : mx;
        mn = v < mn ? v : mn;
    }
    uint64_t run = near_exscan64<kNearThreads, true>(mx, wtot);
    for (int64_t i = a; i < b; ++i) {
        w.pmax[i] = run;
        const uint64_t u = __ldcg(w.umax + i);
        run = u > run ? u : run;
    }
    run = near_exscan64<kNearThreads, false>(mn, wtot);
    for (int64_t i = b - 1; i >= a; --i) {
        w.smin[i] = run;
        const uint64_t v = __ldcg(w.umin + i);
        run = v < run ? v : run;
    }
}

__global__ void __launch_bounds__(kNearThreads) k_near_filter(const uint64_t *__restrict__ keys,
                                                              int64_t n, int64_t nt, NearWs w,
                                                              unsigned long long *stats,
                                                              cudaGraphConditionalHandle cond,
                                                              bool use_cond) {
    __shared__ uint64_t wtot[kNearThreads / 32];
    __shared__ uint32_t wsum[kNearThreads / 32];
    __shared__ int s_first, s_last;
    if (ld_flag(w.ctl)) return;  // gave up: the full sort runs
    const int64_t t = blockIdx.x;
    const int64_t base = t * kNearTile;
    const int own_n = (int)(n - base < kNearTile ? n - base : kNearTile);
    const uint64_t tmin = w.umin[t], tmax = w.umax[t];
    if (!w.dirty[t] && w.pmax[t] <= tmin && w.smin[t] >= tmax) {
        // clean, and within the keys around it: all of it is R
        if (threadIdx.x == 0) {
            w.scnt[t] = 0u;
            w.rkey[t] = tmin;
            w.rpos[t] = (uint32_t)base;
        }
    } else {
        const int j0 = threadIdx.x * kNearItems;
        uint32_t *tile_bits = w.bits + t * kNearWords;
        if (threadIdx.x == 0) s_first = kNearTile;
        const uint32_t marks = my_byte(tile_bits);
        uint64_t k[kNearItems];
        uint64_t hmax = 0ull, hmin = ~0ull;
#pragma unroll
        for (int q = 0; q < kNearItems; ++q) {
            const bool valid = j0 + q < own_n;
            k[q] = valid ? __ldg(keys + base + j0 + q) : 0ull;
            if (valid && !((marks >> q) & 1u)) {
                hmax = k[q] > hmax ? k[q] : hmax;
                hmin = k[q] < hmin ? k[q] : hmin;
            }
        }
        uint64_t pre = near_exscan64<kNearThreads, true>(hmax, wtot);
        uint64_t suf = near_exscan64<kNearThreads, false>(hmin, wtot);
        {
            const uint64_t p = w.pmax[t], s = w.smin[t];
            pre = p > pre ? p : pre;
            suf = s < suf ? s : suf;
        }
        uint32_t sbits = 0;
#pragma unroll
        for (int q = 0; q < kNearItems; ++q) {
            if (j0 + q < own_n) {
                const bool m = (marks >> q) & 1u;
                if (m || k[q] < pre) sbits |= 1u << q;
                if (!m) pre = k[q] > pre ? k[q] : pre;
            }
        }
#pragma unroll
        for (int q = kNearItems - 1; q >= 0; --q) {
            if (j0 + q < own_n) {
                const bool m = (marks >> q) & 1u;
                if (k[q] > suf) sbits |= 1u << q;
                if (!m) suf = k[q] < suf ? k[q] : suf;
            }
        }
        // four threads share a bit word
        uint32_t word = sbits << (j0 & 31);
        word |= __shfl_xor_sync(0xffffffffu, word, 1);
        word |= __shfl_xor_sync(0xffffffffu, word, 2);
        if ((threadIdx.x & 3) == 0) tile_bits[j0 >> 5] = word;
        int first = kNearTile;
#pragma unroll
        for (int q = kNearItems - 1; q >= 0; --q)
            if (j0 + q < own_n && !((sbits >> q) & 1u)) first = j0 + q;
        if (first < kNearTile) atomicMin(&s_first, first);
        const uint32_t cnt = (uint32_t)__popc(sbits);
        const uint32_t ex = near_exsum<kNearThreads>(cnt, wsum);
        if (threadIdx.x == kNearThreads - 1) {
            w.scnt[t] = ex + cnt;
            const int f = s_first;
            if (f < kNearTile) {
                w.rkey[t] = __ldg(keys + base + f);
                w.rpos[t] = (uint32_t)(base + f);
            } else {
                w.rkey[t] = ~0ull;
                w.rpos[t] = kNone;
            }
        }
    }
    if (!last_block(w.ctl + 4, &s_last)) return;
    // offsets of S per tile, and the choice of path
    const int64_t per = (nt + kNearThreads - 1) / kNearThreads;
    const int64_t a = (int64_t)threadIdx.x * per;
    const int64_t b = a + per < nt ? a + per : nt;
    uint32_t sum = 0;
    for (int64_t i = a; i < b; ++i) sum += __ldcg(w.scnt + i);
    uint32_t run = near_exsum<kNearThreads>(sum, wsum);
    for (int64_t i = a; i < b; ++i) {
        w.soff[i] = run;
        run += __ldcg(w.scnt + i);
    }
    if (threadIdx.x == kNearThreads - 1) {
        w.soff[nt] = run;
        w.ctl[2] = (int32_t)run;
        if (run <= (uint32_t)kNearCap) {
            w.ctl[1] = 1;
            if (stats) stats[0] += 1ull;
            // in a CUDA graph: the full sort's conditional node (default: run) is skipped
            if (use_cond) cudaGraphSetConditional(cond, 0u);
        }
    }
}

// first index in the sorted S keys sk/sp[0, m) at or above (k, p)
__device__ __forceinline__ int lower_bound_pairs(const uint64_t *sk, const uint32_t *sp, int lo,
                                                 int hi, uint64_t k, uint32_t p) {
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (pair_less(sk[mid], sp[mid], k, p))
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

__global__ void __launch_bounds__(kNearThreads) k_near_take(const uint64_t *__restrict__ keys,
                                                            int64_t nt, NearWs w) {
    __shared__ uint64_t sk[kNearCap];
    __shared__ uint32_t sp[kNearCap];
    __shared__ uint32_t wsum[kNearThreads / 32];
    __shared__ int s_last;
    if (!ld_flag(w.ctl + 1)) return;
    const int64_t t = blockIdx.x;
    const uint32_t off0 = w.soff[t];
    if (w.soff[t + 1] != off0) {
        const int64_t base = t * kNearTile;
        const int j0 = threadIdx.x * kNearItems;
        const uint32_t sb = my_byte(w.bits + t * kNearWords);
        uint32_t idx = off0 + near_exsum<kNearThreads>((uint32_t)__popc(sb), wsum);
#pragma unroll
        for (int q = 0; q < kNearItems; ++q) {
            if ((sb >> q) & 1u) {
                w.s_key[idx] = __ldg(keys + base + j0 + q);
                w.s_pos[idx] = (uint32_t)(base + j0 + q);
                ++idx;
            }
        }
    }
    if (!last_block(w.ctl + 5, &s_last)) return;
    // S ordered by (key, index): bitonic network over the next power of two
    const int m = w.ctl[2];
    int P = 1;
    while (P < m) P <<= 1;
    for (int i = threadIdx.x; i < P; i += kNearThreads) {
        sk[i] = i < m ? __ldcg(w.s_key + i) : ~0ull;
        sp[i] = i < m ? __ldcg(w.s_pos + i) : kNone;
    }
    __syncthreads();
    for (int k = 2; k <= P; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < P; i += kNearThreads) {
                const int ixj = i ^ j;
                if (ixj > i) {
                    const bool up = (i & k) == 0;
                    const uint64_t ka = sk[i], kb = sk[ixj];
                    const uint32_t pa = sp[i], pb = sp[ixj];
                    if (pair_less(kb, pb, ka, pa) == up) {
                        sk[i] = kb;
                        sk[ixj] = ka;
                        sp[i] = pb;
                        sp[ixj] = pa;
                    }
                }
            }
            __syncthreads();
        }
    }
    for (int i = threadIdx.x; i < m; i += kNearThreads) {
        w.ss_key[i] = sk[i];
        w.ss_pos[i] = sp[i];
    }
    // per tile the S keys it places: from the first R key of the tile (tile 0:
    // from the start) to the first R key of a later tile (or the end)
    for (int64_t u = threadIdx.x; u <= nt; u += kNearThreads) {
        int v;
        if (u == 0) {
            v = 0;
        } else {
            int64_t q = u;
            while (q < nt && w.rpos[q] == kNone) ++q;
            v = q < nt ? lower_bound_pairs(sk, sp, 0, m, w.rkey[q], w.rpos[q]) : m;
        }
        w.tlo[u] = (uint32_t)v;
    }
}

__global__ void __launch_bounds__(kNearThreads) k_near_place(const uint64_t *__restrict__ keys,
                                                             int64_t n, NearWs w,
                                                             uint64_t *__restrict__ keys_out,
                                                             uint32_t *__restrict__ perm_out,
                                                             int32_t *flags, int64_t dest_bias) {
    extern __shared__ __align__(16) unsigned char smem[];
    uint64_t *rk = reinterpret_cast<uint64_t *>(smem);
    uint32_t *rp = reinterpret_cast<uint32_t *>(smem + kNearTile * sizeof(uint64_t));
    __shared__ uint32_t wsum[kNearThreads / 32];
    if (!ld_flag(w.ctl + 1)) return;
    const int64_t t = blockIdx.x;
    const int64_t base = t * kNearTile;
    const int own_n = (int)(n - base < kNearTile ? n - base : kNearTile);
    const int lo = (int)w.tlo[t], hi = (int)w.tlo[t + 1];
    const uint32_t soff = w.soff[t];
    const int s_tile = (int)(w.soff[t + 1] - soff);
    // dest_bias: 0 except under cnb_ctx_inject_sort_faults, which shifts every
    // destination to exercise the destination checks below
    const int64_t r_before = base - (int64_t)soff + dest_bias;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (s_tile == 0 && lo == hi) {
        // every key of the tile is R and no S key falls among them: a shifted copy
        const int64_t shift = r_before + lo - base;
#pragma unroll
        for (int r = 0; r < kNearItems; ++r) {
            const int p = warp * 256 + r * 32 + lane;
            if (p < own_n) {
                const int64_t o = base + p + shift;
                if (o >= 0 && o < n) {
                    keys_out[o] = __ldg(keys + base + p);
                    perm_out[o] = (uint32_t)(base + p);
                } else {
                    set_flag(flags, CNB_FLAG_SORT_CHECK);
                }
            }
        }
        return;
    }
    const int j0 = threadIdx.x * kNearItems;
    const uint32_t sb = my_byte(w.bits + t * kNearWords);
    uint64_t k[kNearItems];
#pragma unroll
    for (int q = 0; q < kNearItems; ++q)
        k[q] = (j0 + q < own_n) ? __ldg(keys + base + j0 + q) : 0ull;
    const uint32_t s_before = near_exsum<kNearThreads>((uint32_t)__popc(sb), wsum);
    // R keys of this tile, compacted in order
    uint32_t r_local = (uint32_t)j0 - s_before;
#pragma unroll
    for (int q = 0; q < kNearItems; ++q) {
        if (j0 + q < own_n && !((sb >> q) & 1u)) {
            rk[r_local] = k[q];
            rp[r_local] = (uint32_t)(base + j0 + q);
            ++r_local;
        }
    }
    __syncthreads();
    r_local = (uint32_t)j0 - s_before;
#pragma unroll
    for (int q = 0; q < kNearItems; ++q) {
        if (j0 + q < own_n && !((sb >> q) & 1u)) {
            const uint32_t pos = (uint32_t)(base + j0 + q);
            int c = lo;
            if (hi - lo <= 16) {
                while (c < hi && pair_less(w.ss_key[c], w.ss_pos[c], k[q], pos)) ++c;
            } else {
                c = lower_bound_pairs(w.ss_key, w.ss_pos, lo, hi, k[q], pos);
            }
            const int64_t o = r_before + r_local + c;
            if (o < n) {
                keys_out[o] = k[q];
                perm_out[o] = pos;
            } else {
                set_flag(flags, CNB_FLAG_SORT_CHECK);
            }
            ++r_local;
        }
    }
    const int r_tile = own_n - s_tile;
    for (int s = lo + threadIdx.x; s < hi; s += kNearThreads) {
        const uint64_t ks = w.ss_key[s];
        const uint32_t ps = w.ss_pos[s];
        const int a = lower_bound_pairs(rk, rp, 0, r_tile, ks, ps);
        const int64_t o = (int64_t)s + r_before + a;
        if (o < n) {
            keys_out[o] = ks;
            perm_out[o] = ps;
        } else {
            set_flag(flags, CNB_FLAG_SORT_CHECK);
        }
    }
}

}  // namespace

int64_t near_bytes(int64_t n_max) {
    const int64_t nt = (n_max + kNearTile - 1) / kNearTile;
    return near_layout(nullptr, nt < 1 ? 1 : nt, nullptr);
}

// Launches the near-sorted path; *skip_full receives the device flag that
// is non-zero when it produced the result (the full sort's kernels then
// return), *never a device flag that stays zero.  use_cond: the launches are
// being captured into a CUDA graph whose conditional node `cond` holds the
// full sort; the path sets it to 0 when it produced the result.
int sort_pairs_near(cnb_ctx *ctx, const uint64_t *keys_in, uint64_t *keys_out,
                    uint32_t *perm_out, int64_t n, cudaStream_t st, const int32_t **skip_full,
                    const int32_t **never, cudaGraphConditionalHandle cond, bool use_cond) {
    const int64_t nt = (n + kNearTile - 1) / kNearTile;
    const int64_t nt_max = (ctx->n_max + kNearTile - 1) / kNearTile;
    NearWs w;
    near_layout(ctx->near, nt_max < 1 ? 1 : nt_max, &w);
    CNB_CUDA(cudaMemsetAsync(w.ctl, 0, 8 * sizeof(int32_t), st));
    CNB_CUDA(cudaFuncSetAttribute(k_near_mark, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)kNearMarkSmem));
    CNB_CUDA(cudaFuncSetAttribute(k_near_place, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)kNearPlaceSmem));
    k_near_mark<<<(unsigned)nt, kNearThreads, kNearMarkSmem, st>>>(keys_in, n, nt, w);
    CNB_TRY(launch_status());
    k_near_filter<<<(unsigned)nt, kNearThreads, 0, st>>>(keys_in, n, nt, w, ctx->sort_stats, cond,
                                                          use_cond);
    CNB_TRY(launch_status());
    k_near_take<<<(unsigned)nt, kNearThreads, 0, st>>>(keys_in, nt, w);
    CNB_TRY(launch_status());
    k_near_place<<<(unsigned)nt, kNearThreads, kNearPlaceSmem, st>>>(keys_in, n, w, keys_out,
                                                                      perm_out, ctx->flags,
                                                                      ctx->near_dest_bias);
    CNB_TRY(launch_status());
    *skip_full = w.ctl + 1;
    *never = w.ctl + 7;  // zeroed with the rest of ctl, never set
    return CNB_OK;
}

}  // namespace cnb
