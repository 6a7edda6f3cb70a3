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
    // grouped traversal scratch (grown on demand by cnb_forces_grouped)
    void *group_scratch = nullptr;
    size_t group_scratch_bytes = 0;
};

namespace cnb {
constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;  // 4096 keys per tile
}  // namespace cnb
