// direct.cu -- float64 minimum-image direct sum on the GPU.
//
// a_i = sum_{j: d2 > 1e-7} G m_j d / (d2 + soft^2)^{3/2}, d = x_j - x_i -
// rint(x_j - x_i) per axis, all float64: the force law of
// src/kernels/physics_kernels.py:118-141 applied to every pair.  Used as the
// accuracy reference of the tree forces and to label opening angles for the
// learned controller.  One 256-thread block per target; sources are read in
// float32 (as stored) and promoted.
#include "common.cuh"

namespace cnb {

__global__ void __launch_bounds__(256) k_direct_f64(const float *__restrict__ px,
                                                    const float *__restrict__ py,
                                                    const float *__restrict__ pz,
                                                    const float *__restrict__ mass, int64_t n,
                                                    const int64_t *__restrict__ targets,
                                                    int64_t nt, double G, double soft2,
                                                    double *__restrict__ out) {
    __shared__ double red[3][8];
    for (int64_t t = blockIdx.x; t < nt; t += gridDim.x) {
        const int64_t i = targets[t];
        const double xi = px[i], yi = py[i], zi = pz[i];
        double ax = 0, ay = 0, az = 0;
        for (int64_t j = threadIdx.x; j < n; j += blockDim.x) {
            double dx = (double)__ldg(px + j) - xi, dy = (double)__ldg(py + j) - yi,
                   dz = (double)__ldg(pz + j) - zi;
            dx -= rint(dx);
            dy -= rint(dy);
            dz -= rint(dz);
            const double d2 = dx * dx + dy * dy + dz * dz;
            if (d2 > 1e-7) {
                const double r = rsqrt(d2 + soft2);
                const double f = (double)__ldg(mass + j) * r * r * r;
                ax += f * dx;
                ay += f * dy;
                az += f * dz;
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            ax += __shfl_xor_sync(0xffffffffu, ax, o);
            ay += __shfl_xor_sync(0xffffffffu, ay, o);
            az += __shfl_xor_sync(0xffffffffu, az, o);
        }
        const int w = threadIdx.x >> 5;
        if ((threadIdx.x & 31) == 0) {
            red[0][w] = ax;
            red[1][w] = ay;
            red[2][w] = az;
        }
        __syncthreads();
        if (threadIdx.x < 3) {
            double s = 0;
            for (int k = 0; k < (int)(blockDim.x >> 5); ++k) s += red[threadIdx.x][k];
            out[3 * t + threadIdx.x] = G * s;
        }
        __syncthreads();
    }
}

}  // namespace cnb

extern "C" int cnb_direct_sum_f64(const float *px, const float *py, const float *pz,
                                  const float *mass, int64_t n, const int64_t *targets,
                                  int64_t n_targets, double G, double soft, double *out,
                                  void *stream) {
    if (n < 0 || n_targets < 0) return CNB_E_INVALID_ARG;
    if (n_targets == 0) return CNB_OK;
    if (!px || !py || !pz || !mass || !targets || !out) return CNB_E_INVALID_ARG;
    const int grid = (int)(n_targets < 148LL * 32 ? n_targets : 148LL * 32);
    cnb::k_direct_f64<<<grid, 256, 0, cnb::as_stream(stream)>>>(px, py, pz, mass, n, targets,
                                                                n_targets, G, soft * soft, out);
    return cnb::launch_status();
}
