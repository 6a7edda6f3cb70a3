// ctx.cuh -- the scratch owner behind cnb_ctx (radix-sort ping-pong buffers
// and per-tile digit counts, grouped-traversal work space).
#pragma once
#include "common.cuh"

struct cnb_ctx {
    int device = 0;
    int64_t n_max = 0;
    int64_t tiles_max = 0;
    uint64_t *keys_tmp[2] = {nullptr, nullptr};
    uint32_t *vals_tmp[2] = {nullptr, nullptr};
    uint32_t *tile_hist = nullptr;  // [256 * (tiles_max + 1)]: digit-major counts, digit totals
                                    // (reduce-then-scan sort of cnb_sort_pairs_noalloc)
    // one-sweep sort: [8 x 256] digit counts of every pass, [8] tile counters,
    // then the look-back words of every pass, [8 x tiles x 256] (2048-key tiles)
    uint32_t *sweep = nullptr;
    int32_t *flags = nullptr;       // CNB_FLAG_* raised by the sort, taken by cnb_ctx_take_flags
    // near-sorted path of the adaptive sort (sort_near.cu): one allocation
    int sort_mode = CNB_SORT_FULL;
    void *near = nullptr;
    unsigned long long *sort_stats = nullptr;  // [near-sorted path taken, full radix sorts run]
    cudaStream_t side = nullptr;    // captures the full sort into a conditional graph node
    // cnb_ctx_inject_sort_faults (tests of the failure paths; off by default):
    int32_t wait_limit = 0;          // look-back polls before a wait gives up (0: 2^22)
    int64_t withheld_tile = -1;      // one-sweep tile that never publishes its counts
    int64_t near_dest_bias = 0;      // added to the near-sorted path's R destinations
    // grouped traversal scratch (grown on demand by cnb_forces_grouped)
    void *group_scratch = nullptr;
    size_t group_scratch_bytes = 0;
};

namespace cnb {
// tiles and the bound on out-of-place keys of the near-sorted path
constexpr int kNearThreads = 512;
constexpr int kNearItems = 8;
constexpr int kNearTile = kNearThreads * kNearItems;  // 4096 keys
constexpr int kNearCap = 2048;                        // at most this many keys leave their run
int64_t near_bytes(int64_t n_max);
int sort_pairs_near(cnb_ctx *ctx, const uint64_t *keys_in, uint64_t *keys_out,
                    uint32_t *perm_out, int64_t n, cudaStream_t st, const int32_t **skip_full,
                    const int32_t **never, cudaGraphConditionalHandle cond, bool use_cond);
int sort_pairs_onesweep(cnb_ctx *ctx, const uint64_t *keys_in, uint64_t *keys_out,
                        const uint32_t *idx_in, uint32_t *perm_out, int64_t n, int key_bits,
                        cudaStream_t st, const int32_t *skip = nullptr);

constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;  // 4096 keys per tile
constexpr int kSweepPasses = 8;                        // 8-bit digits of keys up to 64 bits
constexpr int64_t kSweepMetaWords = kSweepPasses * 256 + 64;  // counts, tile counters, padding
// bytes of the one-sweep scratch for up to n_max keys (tiles of 2048 keys)
// The buffers of one (key, index) sort may be the same array -- keys_in ==
// keys_out or idx_in == perm_out: the sort then runs at least two passes, so
// no pass reads what it writes -- but may not overlap in any other way.
inline bool sort_buffers_ok(const void *keys_in, const void *keys_out, const void *idx_in,
                            const void *perm_out, int64_t n) {
    struct R {
        const char *p;
        int64_t b;
    };
    const R k_in{static_cast<const char *>(keys_in), 8 * n};
    const R k_out{static_cast<const char *>(keys_out), 8 * n};
    const R i_in{static_cast<const char *>(idx_in), idx_in ? 4 * n : 0};
    const R p_out{static_cast<const char *>(perm_out), 4 * n};
    auto overlap = [](R a, R b) { return a.b > 0 && b.b > 0 && a.p < b.p + b.b && b.p < a.p + a.b; };
    if (overlap(k_in, k_out) && k_in.p != k_out.p) return false;
    if (overlap(i_in, p_out) && i_in.p != p_out.p) return false;
    return !overlap(k_in, i_in) && !overlap(k_in, p_out) && !overlap(k_out, i_in) &&
           !overlap(k_out, p_out);
}
inline int64_t sweep_bytes(int64_t n_max) {
    const int64_t tiles = (n_max + 2047) / 2048;
    return kSweepMetaWords * 4 + (int64_t)kSweepPasses * tiles * 256 * 8;
}
}  // namespace cnb
