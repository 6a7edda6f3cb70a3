// sort_noalloc.cu -- cnb_sort_pairs_noalloc: the (key, index) radix sort
// with its scratch in a fixed device array instead of a cnb_ctx.
//
// Some hosts cannot call cudaMalloc on the sort's path: a plugin whose host
// application has reserved the device memory for its own pool, or code that
// runs where an allocation (and the device synchronisation cudaMalloc may
// imply) is not allowed.  For them the scratch lives in the file-scope array
// below, sized for at most CNB_NOALLOC_MAX_KEYS keys.  Every GPU that loads
// libcnb.so holds this array (about 24.3 MiB) until the process exits.
//
// The sort is the reduce-then-scan form (three launches per 8-bit pass: 24
// for 63-bit keys, 12 for 30-bit ones), not the one-sweep sort of
// cnb_sort_pairs; both are stable, so the output is identical.
//
// The array's host-side name is only a stand-in for the device symbol: host
// code must not pass it to a kernel.  The first call on each device looks up
// the device address with cudaGetSymbolAddress (with that device current)
// and caches it for the life of the process; that first call should
// therefore come before any stream capture, and a device reset
// (cudaDeviceReset) after it is not supported: the cached address would
// outlive the module it points into.  All calls share the one array and it
// keeps the last call's contents: nothing in it has to start at zero (each
// pass writes every count it reads), and calls whose work overlaps on the
// GPU -- on different streams, or from different host threads -- race on it.
#include <mutex>

#include "ctx.cuh"

namespace cnb {

int sort_pairs(cnb_ctx *ctx, const uint64_t *keys_in, uint64_t *keys_out,
               const uint32_t *idx_in, uint32_t *perm_out, int64_t n, int key_bits,
               cudaStream_t st);

namespace {
constexpr int64_t kMaxKeys = CNB_NOALLOC_MAX_KEYS;
constexpr int64_t kMaxTiles = (kMaxKeys + kSortTile - 1) / kSortTile;
constexpr size_t kKeyBytes = sizeof(uint64_t) * kMaxKeys;
constexpr size_t kValBytes = sizeof(uint32_t) * kMaxKeys;
constexpr size_t kHistBytes = sizeof(uint32_t) * 256 * (kMaxTiles + 1);  // counts + digit totals
constexpr size_t kScratchBytes = 2 * kKeyBytes + 2 * kValBytes + kHistBytes;

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned char *g_dev_scratch[kMaxDevices] = {};
}  // namespace

static __device__ __align__(256) unsigned char g_sort_scratch[kScratchBytes];

// Device address of g_sort_scratch on the current device (looked up once).
static int scratch_address(unsigned char **out) {
    int dev = 0;
    CNB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return CNB_E_INVALID_ARG;
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_dev_scratch[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_sort_scratch);
        if (e != cudaSuccess || p == nullptr) return record_cuda_error(e != cudaSuccess ? e : cudaErrorInvalidSymbol);
        g_dev_scratch[dev] = static_cast<unsigned char *>(p);
    }
    *out = g_dev_scratch[dev];
    return CNB_OK;
}

}  // namespace cnb

extern "C" int cnb_sort_pairs_noalloc(const uint64_t *keys_in, uint64_t *keys_out,
                                      const uint32_t *idx_in, uint32_t *perm_out, int64_t n,
                                      int key_bits, void *stream) {
    if (n < 0 || key_bits < 1 || key_bits > 64) return CNB_E_INVALID_ARG;
    if (n > cnb::kMaxKeys) return CNB_E_TOO_LARGE;
    if (n == 0) return CNB_OK;
    if (!keys_in || !keys_out || !perm_out) return CNB_E_INVALID_ARG;
    if (!cnb::sort_buffers_ok(keys_in, keys_out, idx_in, perm_out, n)) return CNB_E_INVALID_ARG;
    unsigned char *base = nullptr;
    CNB_TRY(cnb::scratch_address(&base));
    // a view of the fixed array shaped like a context: nothing is allocated
    cnb_ctx view;
    view.n_max = cnb::kMaxKeys;
    view.tiles_max = cnb::kMaxTiles;
    view.keys_tmp[0] = reinterpret_cast<uint64_t *>(base);
    view.keys_tmp[1] = reinterpret_cast<uint64_t *>(base + cnb::kKeyBytes);
    view.vals_tmp[0] = reinterpret_cast<uint32_t *>(base + 2 * cnb::kKeyBytes);
    view.vals_tmp[1] = reinterpret_cast<uint32_t *>(base + 2 * cnb::kKeyBytes + cnb::kValBytes);
    view.tile_hist = reinterpret_cast<uint32_t *>(base + 2 * cnb::kKeyBytes + 2 * cnb::kValBytes);
    return cnb::sort_pairs(&view, keys_in, keys_out, idx_in, perm_out, n, key_bits,
                           cnb::as_stream(stream));
}
