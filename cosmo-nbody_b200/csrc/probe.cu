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
// The same with packed float2 FMAs (FFMA2, two FMAs per instruction), as the
// traversal's force loops issue them: flops = 2 * 2 * 8 * iters * threads.
__global__ void __launch_bounds__(256) k_fma2_probe(float *out, int64_t iters, float a, float b) {
    float2 v[8];
    const float2 a2 = make_float2(a, a), b2 = make_float2(b, b);
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = make_float2(threadIdx.x * 1e-3f + k, threadIdx.x * 2e-3f - k);
    for (int64_t it = 0; it < iters; ++it) {
#pragma unroll
        for (int k = 0; k < 8; ++k) v[k] = __ffma2_rn(v[k], a2, b2);
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += v[k].x + v[k].y;
    out[blockIdx.x * (int64_t)blockDim.x + threadIdx.x] = s;
}
}  // namespace cnb

extern "C" int cnb_fma2_probe(float *out, int64_t iters, int blocks, void *stream) {
    if (!out || iters < 1 || blocks < 1) return CNB_E_INVALID_ARG;
    cnb::k_fma2_probe<<<blocks, 256, 0, cnb::as_stream(stream)>>>(out, iters, 0.999999f, 1e-6f);
    return cnb::launch_status();
}

extern "C" int cnb_fma_probe(float *out, int64_t iters, int blocks, void *stream) {
    if (!out || iters < 1 || blocks < 1) return CNB_E_INVALID_ARG;
    cnb::k_fma_probe<<<blocks, 256, 0, cnb::as_stream(stream)>>>(out, iters, 0.999999f, 1e-6f);
    return cnb::launch_status();
}
