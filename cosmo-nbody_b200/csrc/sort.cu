// sort.cu -- stable LSD radix sort of (Morton key, index) pairs and the
// permutation gathers (src/core/state.py:20-40: cp.argsort + 8 gathers).
//
// One pass per 8-bit digit, reduce-then-scan (no inter-block waiting):
//   k_digit_count   per-tile digit counts (shared-memory histograms)
//   k_scan_rows     exclusive scan of each digit's tile counts (one block
//                   per digit) and the digit totals
//   k_scatter       stable in-tile ranks (warp __match_any_sync + per-warp
//                   digit counters), the tile reordered by digit in shared
//                   memory, then coalesced runs written to global positions
// A 4096-key tile per 256-thread block keeps one pass at 8 B read for the
// count, 12 B read + 12 B written for the scatter, per key.
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
    if (passes == 1 && keys_in == keys_out) passes = 2;
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
    if (e == cudaSuccess) e = cudaMalloc(&c->tile_hist, sizeof(uint32_t) * 256 * (c->tiles_max + 1));
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
    return cnb::sort_pairs(ctx, keys_in, keys_out, idx_in, perm_out, n, key_bits,
                           cnb::as_stream(stream));
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
