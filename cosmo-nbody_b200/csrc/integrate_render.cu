// integrate_render.cu -- Hubble-drag kick/drift (physics_kernels.py:155-203)
// and the MVP density splat (render_kernels.py:12-47).
#include "common.cuh"

namespace cnb {

// physics_kernels.py:155-203: float64 kick and drift of float32 state, wrap
// by x - floor(x).  Explicit round-to-nearest operations (no contraction) so
// the result is the same on every compiler.
__global__ void __launch_bounds__(256) k_integrate(float *__restrict__ px, float *__restrict__ py,
                                                   float *__restrict__ pz, float *__restrict__ vx,
                                                   float *__restrict__ vy, float *__restrict__ vz,
                                                   const float *__restrict__ force, int64_t n,
                                                   double drag, double f_scale, double dt,
                                                   double drift) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        float *pp[3] = {px, py, pz};
        float *vv[3] = {vx, vy, vz};
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            double v = __dadd_rn(__dmul_rn((double)vv[k][i], drag),
                                 __dmul_rn(__dmul_rn((double)__ldg(force + 3 * i + k), f_scale), dt));
            vv[k][i] = __double2float_rn(v);
            double p = __dadd_rn((double)pp[k][i], __dmul_rn(__dmul_rn(v, dt), drift));
            p = __dsub_rn(p, floor(p));
            pp[k][i] = __double2float_rn(p);
        }
    }
}

// ---------------------------------------------------------------- splat

// render_kernels.py:24-42: clip coordinates as float32 sums of float32
// products, w test / 1.0 / w / screen mapping in float64.  Returns the flat
// pixel index and the float32 weight 2.5 / w, or -1.
__device__ __forceinline__ int64_t splat_pixel(const float *m, float x, float y, float z,
                                               int width, int height, float *val) {
    float xc = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(m[0], x), __fmul_rn(m[1], y)),
                                   __fmul_rn(m[2], z)), m[3]);
    float yc = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(m[4], x), __fmul_rn(m[5], y)),
                                   __fmul_rn(m[6], z)), m[7]);
    float wc = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(m[12], x), __fmul_rn(m[13], y)),
                                   __fmul_rn(m[14], z)), m[15]);
    if (!((double)wc > 0.01)) return -1;
    double inv = __ddiv_rn(1.0, (double)wc);
    double sx = __dmul_rn(__dmul_rn(__dadd_rn(__dmul_rn((double)xc, inv), 1.0), 0.5), (double)width);
    double sy = __dmul_rn(__dmul_rn(__dsub_rn(1.0, __dmul_rn((double)yc, inv)), 0.5), (double)height);
    if (!(0.0 <= sx && sx < (double)width && 0.0 <= sy && sy < (double)height)) return -1;
    *val = __double2float_rn(__dmul_rn(2.5, inv));
    return (int64_t)sy * width + (int64_t)sx;
}

constexpr int kSplatThreads = 256;
constexpr int kSplatItems = 8;                    // particles per thread
constexpr int kSplatTilePix = 12160;              // 47.5 KB shared-memory tile

// Tile-privatised splat.  Each block takes kSplatThreads*kSplatItems
// consecutive particles; after a Morton sort they project to a compact
// screen region.  If the block's pixel bounding box fits kSplatTilePix, the
// block accumulates in shared memory and adds each touched pixel to the
// global grid once; otherwise it adds per particle to the global grid.
__global__ void __launch_bounds__(kSplatThreads) k_splat(const float *__restrict__ px,
                                                         const float *__restrict__ py,
                                                         const float *__restrict__ pz,
                                                         float *__restrict__ grid, const float *__restrict__ mvp,
                                                         int64_t n, int width, int height) {
    __shared__ float tile[kSplatTilePix];
    __shared__ int bb[4];
    __shared__ float m[16];
    if (threadIdx.x < 16) m[threadIdx.x] = mvp[threadIdx.x];
    if (threadIdx.x == 0) {
        bb[0] = INT32_MAX; bb[1] = INT32_MAX; bb[2] = -1; bb[3] = -1;
    }
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kSplatThreads * kSplatItems;
    int64_t pix[kSplatItems];
    float val[kSplatItems];
    int x0 = INT32_MAX, y0 = INT32_MAX, x1 = -1, y1 = -1;
#pragma unroll
    for (int r = 0; r < kSplatItems; ++r) {
        int64_t i = base + (int64_t)r * kSplatThreads + threadIdx.x;
        pix[r] = -1;
        if (i < n) pix[r] = splat_pixel(m, __ldcs(px + i), __ldcs(py + i), __ldcs(pz + i), width,
                                        height, &val[r]);
        if (pix[r] >= 0) {
            int sy = (int)(pix[r] / width), sx = (int)(pix[r] - (int64_t)sy * width);
            x0 = min(x0, sx); x1 = max(x1, sx); y0 = min(y0, sy); y1 = max(y1, sy);
        }
    }
    // block bounding box of touched pixels
    for (int o = 16; o > 0; o >>= 1) {
        x0 = min(x0, __shfl_xor_sync(0xffffffffu, x0, o));
        y0 = min(y0, __shfl_xor_sync(0xffffffffu, y0, o));
        x1 = max(x1, __shfl_xor_sync(0xffffffffu, x1, o));
        y1 = max(y1, __shfl_xor_sync(0xffffffffu, y1, o));
    }
    if ((threadIdx.x & 31) == 0 && x1 >= 0) {
        atomicMin(&bb[0], x0); atomicMin(&bb[1], y0);
        atomicMax(&bb[2], x1); atomicMax(&bb[3], y1);
    }
    __syncthreads();
    if (bb[2] < 0) return;  // nothing visible
    const int bw = bb[2] - bb[0] + 1, bh = bb[3] - bb[1] + 1;
    if ((int64_t)bw * bh > kSplatTilePix) {
#pragma unroll
        for (int r = 0; r < kSplatItems; ++r)
            if (pix[r] >= 0) atomicAdd(grid + pix[r], val[r]);
        return;
    }
    const int area = bw * bh;
    for (int k = threadIdx.x; k < area; k += kSplatThreads) tile[k] = 0.f;
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kSplatItems; ++r) {
        if (pix[r] >= 0) {
            int sy = (int)(pix[r] / width), sx = (int)(pix[r] - (int64_t)sy * width);
            atomicAdd(&tile[(sy - bb[1]) * bw + (sx - bb[0])], val[r]);
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < area; k += kSplatThreads) {
        float v = tile[k];
        if (v != 0.f) {
            int ty = k / bw, tx = k - ty * bw;
            atomicAdd(grid + (int64_t)(bb[1] + ty) * width + (bb[0] + tx), v);
        }
    }
}

}  // namespace cnb

using namespace cnb;

extern "C" int cnb_integrate(float *px, float *py, float *pz, float *vx, float *vy, float *vz,
                             const float *force, int64_t n, double a, double H, double dt,
                             void *stream) {
    if (n < 0) return CNB_E_INVALID_ARG;
    if (n == 0) return CNB_OK;
    if (!px || !py || !pz || !vx || !vy || !vz || !force) return CNB_E_INVALID_ARG;
    const double drag = 1.0 - (H * dt);
    const double f_scale = 1.0 / a;
    const double drift = 1.0 / a;
    k_integrate<<<grid_for(n, 256, 148 * 16), 256, 0, as_stream(stream)>>>(
        px, py, pz, vx, vy, vz, force, n, drag, f_scale, dt, drift);
    return launch_status();
}

extern "C" int cnb_render_density(const float *px, const float *py, const float *pz,
                                  float *grid, const float *mvp, int64_t n, int width,
                                  int height, void *stream) {
    if (n < 0 || width <= 0 || height <= 0) return CNB_E_INVALID_ARG;
    if (n == 0) return CNB_OK;
    if (!px || !py || !pz || !grid || !mvp) return CNB_E_INVALID_ARG;
    const int64_t per_block = (int64_t)kSplatThreads * kSplatItems;
    const int64_t blocks = (n + per_block - 1) / per_block;
    if (blocks > INT32_MAX) return CNB_E_TOO_LARGE;
    k_splat<<<(unsigned)blocks, kSplatThreads, 0, as_stream(stream)>>>(px, py, pz, grid, mvp, n,
                                                                      width, height);
    return launch_status();
}
