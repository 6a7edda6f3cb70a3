// capi.cu -- library-wide entry points (version, errors, launch counter).
#include <atomic>

#include "common.cuh"

namespace cnb {
static thread_local int g_last_cuda_error = 0;
static std::atomic<int64_t> g_launches{0};

int record_cuda_error(cudaError_t e) {
    g_last_cuda_error = (int)e;
    return CNB_E_CUDA;
}
void count_launch(int k) { g_launches.fetch_add(k, std::memory_order_relaxed); }
}  // namespace cnb

extern "C" int cnb_version(void) { return 1; }

extern "C" int cnb_last_cuda_error(void) { return cnb::g_last_cuda_error; }

extern "C" int64_t cnb_launch_count(void) {
    return cnb::g_launches.load(std::memory_order_relaxed);
}

extern "C" const char *cnb_error_string(int code) {
    switch (code) {
        case CNB_OK: return "ok";
        case CNB_E_INVALID_ARG: return "invalid argument";
        case CNB_E_CUDA: return "CUDA error";
        case CNB_E_NO_MEMORY: return "out of device memory";
        case CNB_E_TOO_LARGE: return "size exceeds the supported maximum";
        case CNB_E_DEVICE_FLAG: return "device reported an error flag";
        default: return "unknown error";
    }
}
