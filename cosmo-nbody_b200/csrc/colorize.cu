// colorize.cu -- density grid -> RGB frame (src/utils/visualizer.py:115-171)
// in two kernels instead of ~20 elementwise launches: a max reduction of
// log1p(120 g), then one pass doing normalisation, gamma 2.2, the four-band
// colour map, the x1.3 gain, the clip and (optionally) the 8-bit packing of
// src/core/engine.py:139.  float32 throughout, as the reference's CuPy code.
#include "common.cuh"

namespace cnb {

__global__ void __launch_bounds__(256) k_log_max(const float *__restrict__ grid, int64_t n,
                                                 unsigned int *__restrict__ max_bits) {
    float m = 0.f;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        m = fmaxf(m, log1pf(grid[i] * 120.0f));
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    // non-negative floats order like their bit patterns
    if ((threadIdx.x & 31) == 0) atomicMax(max_bits, __float_as_uint(m));
}

__global__ void __launch_bounds__(256) k_colorize(const float *__restrict__ grid, int64_t n,
                                                  const unsigned int *__restrict__ max_bits,
                                                  float *__restrict__ rgb,
                                                  unsigned char *__restrict__ rgb8) {
    const float denom = __uint_as_float(*max_bits) + 1e-9f;
    const float T1 = 0.6f, T2 = 0.72f, T3 = 0.82f;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const float img = log1pf(grid[i] * 120.0f) / denom;
        const float val = powf(img, 2.2f);
        float r = 0.f, g = 0.f, b = 0.f;
        if (val <= T1) {
            b = (val / T1) * 0.8f;
        } else if (val <= T2) {
            const float t = (val - T1) / (T2 - T1);
            b = (1.0f - t) * 0.8f;
            g = t * 0.9f;
        } else if (val <= T3) {
            const float t = (val - T2) / (T3 - T2);
            g = 0.9f + t * 0.1f;
            r = t;
        } else {
            const float t = (val - T3) / (1.0f - T3);
            r = 1.0f;
            g = 1.0f - t;
        }
        r = fminf(fmaxf(r * 1.3f, 0.f), 1.f);
        g = fminf(fmaxf(g * 1.3f, 0.f), 1.f);
        b = fminf(fmaxf(b * 1.3f, 0.f), 1.f);
        if (rgb) {
            rgb[3 * i] = r;
            rgb[3 * i + 1] = g;
            rgb[3 * i + 2] = b;
        }
        if (rgb8) {  // (frame * 255).astype(uint8): truncation
            rgb8[3 * i] = (unsigned char)(r * 255.0f);
            rgb8[3 * i + 1] = (unsigned char)(g * 255.0f);
            rgb8[3 * i + 2] = (unsigned char)(b * 255.0f);
        }
    }
}

}  // namespace cnb

extern "C" int cnb_colorize(const float *grid, int width, int height, float *rgb,
                            unsigned char *rgb8, unsigned int *scratch, void *stream) {
    if (width <= 0 || height <= 0 || !grid || !scratch || (!rgb && !rgb8)) return CNB_E_INVALID_ARG;
    const int64_t n = (int64_t)width * height;
    cudaStream_t st = cnb::as_stream(stream);
    CNB_CUDA(cudaMemsetAsync(scratch, 0, sizeof(unsigned int), st));
    cnb::k_log_max<<<cnb::grid_for(n, 256, 148 * 8), 256, 0, st>>>(grid, n, scratch);
    CNB_TRY(cnb::launch_status());
    cnb::k_colorize<<<cnb::grid_for(n, 256, 148 * 16), 256, 0, st>>>(grid, n, scratch, rgb, rgb8);
    return cnb::launch_status();
}
