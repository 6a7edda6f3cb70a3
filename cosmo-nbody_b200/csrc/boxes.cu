// boxes.cu -- many independent periodic boxes in one tree (no reference
// counterpart; the reference simulates one box).
//
// Every body carries its box id in the top bits of its key:
//   key = box << (3L) | morton_L(x, y, z),  L = (63 - box_bits) / 3,
// with coordinates in the box's own unit cube.  One sort orders all boxes,
// one Karras build makes each box's bodies one subtree (the keys of a box
// share a prefix no other key has), so the upward pass runs unchanged and
// the traversal of a bucket starts at its box's subtree root.
#include "common.cuh"

namespace cnb {

__device__ __forceinline__ uint64_t spread_bits3(uint64_t v, int L) {
    uint64_t r = 0;
    for (int b = 0; b < L; ++b) r |= ((v >> b) & 1ull) << (3 * b);
    return r;
}

__global__ void __launch_bounds__(256) k_codes_boxes(const float *__restrict__ x,
                                                     const float *__restrict__ y,
                                                     const float *__restrict__ z,
                                                     const int32_t *__restrict__ box,
                                                     uint64_t *__restrict__ codes, int64_t n,
                                                     int L) {
    const double scale = (double)(1ull << L);
    const uint64_t lim = (1ull << L) - 1;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        uint64_t c[3];
        const float p[3] = {x[i], y[i], z[i]};
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const double s = (double)p[k] * scale;
            uint64_t v = (s > 0.0) ? (uint64_t)s : 0ull;
            c[k] = v > lim ? lim : v;
        }
        codes[i] = ((uint64_t)box[i] << (3 * L)) | spread_bits3(c[0], L) |
                   (spread_bits3(c[1], L) << 1) | (spread_bits3(c[2], L) << 2);
    }
}

// Subtree root of each box: the node whose body range lies in one box while
// its parent's does not (or that has no parent).
__global__ void __launch_bounds__(256) k_box_roots(const int2 *__restrict__ ranges,
                                                   const int32_t *__restrict__ parents,
                                                   const uint64_t *__restrict__ codes, int shift,
                                                   int64_t n, int n_boxes,
                                                   int32_t *__restrict__ roots) {
    const int64_t m = 2 * n - 1;
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < m;
         v += (int64_t)gridDim.x * blockDim.x) {
        int lo, hi;
        if (v < n) {
            lo = hi = (int)v;
        } else {
            const int2 r = ranges[v - n];
            lo = r.x;
            hi = r.y;
        }
        const uint64_t b = codes[lo] >> shift;
        if ((codes[hi] >> shift) != b) continue;
        const int32_t p = parents[v];
        bool top = p < 0;
        if (!top) {
            const int2 pr = ranges[p - n];
            top = (codes[pr.x] >> shift) != b || (codes[pr.y] >> shift) != b;
        }
        if (top && b < (uint64_t)n_boxes) roots[b] = (int32_t)v;
    }
}

// physics_kernels.py:155-203 integrate with per-box (a, H, dt) taken from
// box_aHdt[3 * box] (float64), box = key >> shift.
__global__ void __launch_bounds__(256) k_integrate_boxes(float *__restrict__ px, float *__restrict__ py,
                                                         float *__restrict__ pz, float *__restrict__ vx,
                                                         float *__restrict__ vy, float *__restrict__ vz,
                                                         const float *__restrict__ force,
                                                         const uint64_t *__restrict__ codes,
                                                         int shift, int64_t n,
                                                         const double *__restrict__ box_aHdt) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t b = codes[i] >> shift;
        const double a = box_aHdt[3 * b], H = box_aHdt[3 * b + 1], dt = box_aHdt[3 * b + 2];
        const double drag = 1.0 - (H * dt), f_scale = 1.0 / a, drift = 1.0 / a;
        float *pp[3] = {px, py, pz};
        float *vv[3] = {vx, vy, vz};
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const double v = __dadd_rn(__dmul_rn((double)vv[k][i], drag),
                                       __dmul_rn(__dmul_rn((double)force[3 * i + k], f_scale), dt));
            vv[k][i] = __double2float_rn(v);
            double p = __dadd_rn((double)pp[k][i], __dmul_rn(__dmul_rn(v, dt), drift));
            p = __dsub_rn(p, floor(p));
            pp[k][i] = __double2float_rn(p);
        }
    }
}

}  // namespace cnb

using namespace cnb;

extern "C" int cnb_compute_codes_boxes(const float *x, const float *y, const float *z,
                                       const int32_t *box, uint64_t *codes, int64_t n,
                                       int box_bits, void *stream) {
    if (n < 0 || box_bits < 0 || box_bits > 30) return CNB_E_INVALID_ARG;
    if (n == 0) return CNB_OK;
    if (!x || !y || !z || !box || !codes) return CNB_E_INVALID_ARG;
    const int L = (63 - box_bits) / 3;
    k_codes_boxes<<<grid_for(n, 256), 256, 0, as_stream(stream)>>>(x, y, z, box, codes, n, L);
    return launch_status();
}

extern "C" int cnb_box_roots(const int32_t *ranges, const int32_t *parents,
                             const uint64_t *codes, int box_bits, int64_t n, int n_boxes,
                             int32_t *roots, void *stream) {
    if (n < 2 || box_bits < 0 || box_bits > 30 || n_boxes < 1) return CNB_E_INVALID_ARG;
    if (!ranges || !parents || !codes || !roots) return CNB_E_INVALID_ARG;
    const int shift = 3 * ((63 - box_bits) / 3);
    cudaStream_t st = as_stream(stream);
    CNB_CUDA(cudaMemsetAsync(roots, 0xff, sizeof(int32_t) * n_boxes, st));
    k_box_roots<<<grid_for(2 * n - 1, 256), 256, 0, st>>>(reinterpret_cast<const int2 *>(ranges),
                                                          parents, codes, shift, n, n_boxes, roots);
    return launch_status();
}

extern "C" int cnb_integrate_boxes(float *px, float *py, float *pz, float *vx, float *vy,
                                   float *vz, const float *force, const uint64_t *codes,
                                   int box_bits, int64_t n, const double *box_aHdt, void *stream) {
    if (n < 0 || box_bits < 0 || box_bits > 30) return CNB_E_INVALID_ARG;
    if (n == 0) return CNB_OK;
    if (!px || !py || !pz || !vx || !vy || !vz || !force || !codes || !box_aHdt)
        return CNB_E_INVALID_ARG;
    const int shift = 3 * ((63 - box_bits) / 3);
    k_integrate_boxes<<<grid_for(n, 256, 148 * 16), 256, 0, as_stream(stream)>>>(
        px, py, pz, vx, vy, vz, force, codes, shift, n, box_aHdt);
    return launch_status();
}
