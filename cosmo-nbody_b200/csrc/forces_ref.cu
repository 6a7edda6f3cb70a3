// forces_ref.cu -- per-particle stack traversal with the reference's
// opening test (src/kernels/physics_kernels.py:14-153).
//
// One thread per target, depth-first, 64-entry stack.  Node order, the
// opening test (x-extent, clamped to `box` above box/2, against theta^2 d^2
// with d the per-axis minimum image of the CoM) and the silent drop of both
// children when fewer than two stack slots remain are the reference's; the
// drop is also reported as CNB_FLAG_STACK_OVERFLOW.
//
// T = double follows the float64 arithmetic compiled Numba gives the
// reference (float32 node data, `round()` promoting the displacement);
// T = float is the float32 form.  The reference's shared-memory copy of the
// top 256 nodes only mirrors node data and is not needed for the result.
#include "common.cuh"

namespace cnb {

template <typename T>
struct RefMath;

template <>
struct RefMath<double> {
    // dx -= round(dx): float32 difference, rint in float64, result float64.
    static __device__ __forceinline__ double wrap(float d) {
        return (double)d - rint((double)d);
    }
    static __device__ __forceinline__ double inv_r3(double d2, double soft2) {
        double d_inv = 1.0 / sqrt(d2 + soft2);
        return d_inv * d_inv * d_inv;
    }
};

template <>
struct RefMath<float> {
    static __device__ __forceinline__ float wrap(float d) { return d - rintf(d); }
    static __device__ __forceinline__ float inv_r3(float d2, float soft2) {
        float d_inv = rsqrtf(d2 + soft2);
        return d_inv * d_inv * d_inv;
    }
};

template <typename T>
__global__ void __launch_bounds__(128) k_forces_ref(
    const float *__restrict__ px, const float *__restrict__ py, const float *__restrict__ pz,
    const int2 *__restrict__ children, const float *__restrict__ n_mass,
    const float *__restrict__ n_com, const float *__restrict__ n_min,
    const float *__restrict__ n_max, float *__restrict__ force, T theta_sq, T G, T soft2, T box,
    const int32_t *__restrict__ root_idx, int64_t off, int64_t count, int64_t n,
    int32_t *status) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= count) return;
    const int64_t i = off + t;
    if (i >= n) return;
    const int64_t m_nodes = 2 * n - 1;
    const float x = px[i], y = py[i], z = pz[i];
    if (!(isfinite(x) && isfinite(y) && isfinite(z))) set_flag(status, CNB_FLAG_NONFINITE);
    T ax = 0, ay = 0, az = 0;
    int32_t stack[64];
    int top = 0;
    stack[top++] = __ldg(root_idx);
    bool overflow = false, bad = false;
    const T half_box = box * (T)0.5;
    int64_t visits = 0;
    while (top > 0) {
        // a valid tree visits every node at most once per target
        if (++visits > m_nodes) {
            bad = true;
            break;
        }
        const int32_t node = stack[--top];
        if (node < 0 || node >= m_nodes) {
            bad = true;
            continue;
        }
        const float nm = __ldg(n_mass + node);
        if (nm <= 0.f) continue;
        const float cx = __ldg(n_com + 3 * node), cy = __ldg(n_com + 3 * node + 1),
                    cz = __ldg(n_com + 3 * node + 2);
        const int2 ch = __ldg(children + node);
        const T dx = RefMath<T>::wrap(cx - x);
        const T dy = RefMath<T>::wrap(cy - y);
        const T dz = RefMath<T>::wrap(cz - z);
        const T d2 = dx * dx + dy * dy + dz * dz;
        bool use_node = (ch.x == -1);
        if (!use_node) {
            const float sxf = __ldg(n_max + 3 * node) - __ldg(n_min + 3 * node);
            const T sx = ((T)sxf > half_box) ? box : (T)sxf;
            use_node = (sx * sx) < (theta_sq * d2);
        }
        if (use_node) {
            if (d2 > (T)1e-7) {
                const T f = G * (T)nm * RefMath<T>::inv_r3(d2, soft2);
                ax += f * dx;
                ay += f * dy;
                az += f * dz;
            }
        } else if (top + 1 < 64) {
            if (ch.x != -1) stack[top++] = ch.y;
            if (ch.y != -1) stack[top++] = ch.x;
        } else {
            overflow = true;
        }
    }
    const float fx = (float)ax, fy = (float)ay, fz = (float)az;
    force[3 * i] = fx;
    force[3 * i + 1] = fy;
    force[3 * i + 2] = fz;
    if (overflow) set_flag(status, CNB_FLAG_STACK_OVERFLOW);
    if (bad) set_flag(status, CNB_FLAG_BAD_TOPOLOGY);
    if (!isfinite(fx) || !isfinite(fy) || !isfinite(fz)) set_flag(status, CNB_FLAG_NONFINITE);
}

}  // namespace cnb

using namespace cnb;

extern "C" int cnb_compute_forces(const float *px, const float *py, const float *pz,
                                  const int32_t *children, const float *n_mass,
                                  const float *n_com, const float *n_min, const float *n_max,
                                  float *force, double theta, double G, double soft, double box,
                                  const int32_t *root_idx, int64_t off, int64_t count, int64_t n,
                                  int precision, int32_t *status, void *stream) {
    if (n < 0 || off < 0 || count < 0) return CNB_E_INVALID_ARG;
    if (count == 0 || off >= n) return CNB_OK;
    if (!px || !py || !pz || !children || !n_mass || !n_com || !n_min || !n_max || !force ||
        !root_idx)
        return CNB_E_INVALID_ARG;
    if ((reinterpret_cast<uintptr_t>(children) & 7) != 0) return CNB_E_INVALID_ARG;
    if (2 * n - 1 > (int64_t)INT32_MAX) return CNB_E_TOO_LARGE;
    if (count > n - off) count = n - off;
    cudaStream_t st = as_stream(stream);
    const int block = 128;
    const int64_t grid = (count + block - 1) / block;
    if (grid > INT32_MAX) return CNB_E_TOO_LARGE;
    const int2 *ch = reinterpret_cast<const int2 *>(children);
    if (precision == CNB_PREC_F64) {
        k_forces_ref<double><<<(unsigned)grid, block, 0, st>>>(
            px, py, pz, ch, n_mass, n_com, n_min, n_max, force, theta * theta, G, soft * soft,
            box, root_idx, off, count, n, status);
    } else if (precision == CNB_PREC_F32) {
        k_forces_ref<float><<<(unsigned)grid, block, 0, st>>>(
            px, py, pz, ch, n_mass, n_com, n_min, n_max, force, (float)(theta * theta), (float)G,
            (float)(soft * soft), (float)box, root_idx, off, count, n, status);
    } else {
        return CNB_E_INVALID_ARG;
    }
    return launch_status();
}
