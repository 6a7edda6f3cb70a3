// common.cuh -- shared helpers of libcnb.so (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "cnb.h"

namespace cnb {

constexpr int kSMs = 148;  // B200

// Records the last CUDA error for cnb_last_cuda_error() and maps it to CNB_E_CUDA.
int record_cuda_error(cudaError_t e);
void count_launch(int k = 1);

inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

// Checks the launch that was just issued.
inline int launch_status() {
    count_launch();
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? CNB_OK : record_cuda_error(e);
}

inline int grid_for(int64_t n, int block, int64_t cap = 148LL * 64) {
    int64_t g = (n + block - 1) / block;
    if (g < 1) g = 1;
    if (g > cap) g = cap;
    return (int)g;
}

__device__ __forceinline__ void set_flag(int32_t *status, int32_t bit) {
    if (status) atomicOr(status, bit);
}

// Device-scope atomic add with acquire-release semantics: the caller's
// earlier stores are visible to whoever observes the increment (release),
// and stores that other threads released before their increments are
// visible to the caller's later loads (acquire).  One instruction in place of
// fence + atomicAdd + fence.
__device__ __forceinline__ int32_t atomic_add_acq_rel(int32_t *addr, int32_t v) {
    int32_t old;
    asm volatile("atom.acq_rel.gpu.global.add.s32 %0, [%1], %2;"
                 : "=r"(old)
                 : "l"(addr), "r"(v)
                 : "memory");
    return old;
}

}  // namespace cnb

#define CNB_TRY(expr)                   \
    do {                                \
        int _rc = (expr);               \
        if (_rc != CNB_OK) return _rc;  \
    } while (0)

#define CNB_CUDA(expr)                                              \
    do {                                                            \
        cudaError_t _e = (expr);                                    \
        if (_e != cudaSuccess) return cnb::record_cuda_error(_e);   \
    } while (0)
