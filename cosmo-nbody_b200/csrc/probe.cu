// probe.cu -- FP32 FMA throughput probe: the denominator of the traversal's
// roofline (no reference counterpart).  Each thread runs 8 independent FMA
// chains for `iters` rounds; one result per thread is stored so nothing is
// eliminated.  flops = 2 * 8 * iters * threads.
#include "common.cuh"

namespace cnb {
__global__ void __launch_bounds__(256) k_fma_probe(float *out, int64_t iters, float a, float b) {
    float v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = threadIdx.x * 1e-3f + k;
    for (int64_t it = 0; it < iters; ++it) {
#pragma unroll
        for (int k = 0; k < 8; ++k) v[k] = fmaf(v[k], a, b);
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += v[k];
    out[blockIdx.x * (int64_t)blockDim.x + threadIdx.x] = s;
}
}  // namespace cnb

extern "C" int cnb_fma_probe(float *out, int64_t iters, int blocks, void *stream) {
    if (!out || iters < 1 || blocks < 1) return CNB_E_INVALID_ARG;
    cnb::k_fma_probe<<<blocks, 256, 0, cnb::as_stream(stream)>>>(out, iters, 0.999999f, 1e-6f);
    return cnb::launch_status();
}
