// ewald.cu -- periodic (Ewald) force law support (no reference counterpart:
// the reference applies the minimum-image force, physics_kernels.py:118-141).
//
// Unit box, G = 1, unit source mass, d = source - target.  The acceleration
// towards a point mass and all its periodic images, with the uniform
// neutralising background of the Ewald convention, is
//   f_per(d) = sum_n d_n / r_n^3 [erfc(a r_n) + 2 a r_n / sqrt(pi) exp(-a^2 r_n^2)]
//            + 4 pi sum_{k != 0} k / k^2 exp(-k^2 / 4 a^2) sin(k . d),
// d_n = d - n, k = 2 pi m.  Near d = 0, f_per(d) = d / |d|^3 - (4 pi / 3) d
// + g(d) with g smooth, odd and O(|d|^3).
//
// cnb_ewald_table tabulates g, its Jacobian and its second derivatives on
// the octant [0, 1/2]^3 in
// float64 arithmetic (stored as float32); the grouped traversal's "ewald"
// test reads it.  cnb_direct_sum_ewald_f64 is the float64 accuracy oracle:
// every pair's periodic force to float64 precision.
#include <math.h>

#include "common.cuh"

namespace cnb {

constexpr double kAlpha = 2.0;
constexpr int kReal = 3;   // real-space images |n_i| <= 3, those within r = 3 summed
constexpr int kRecip = 3;  // reciprocal vectors |m_i| <= 3, those with |m|^2 <= 12 summed
constexpr double kPi = 3.14159265358979323846;

// B(r) = erfc(a r) + 2 a r / sqrt(pi) exp(-a^2 r^2) and B'(r).
__device__ __forceinline__ void ewald_b(double r, double &b, double &db) {
    const double e = exp(-kAlpha * kAlpha * r * r);
    b = erfc(kAlpha * r) + 2.0 * kAlpha * r / sqrt(kPi) * e;
    db = -4.0 * kAlpha * kAlpha * kAlpha * r * r / sqrt(kPi) * e;
}

// f_per(d) (without_mono: minus d/|d|^3) and, if jac != null, its Jacobian
// d f_i / d d_j as (xx, xy, xz, yy, yz, zz).
__device__ void ewald_force(const double d[3], bool without_mono, double f[3], double *jac) {
    f[0] = f[1] = f[2] = 0.0;
    double J[6] = {0, 0, 0, 0, 0, 0};
    for (int nx = -kReal; nx <= kReal; ++nx)
        for (int ny = -kReal; ny <= kReal; ++ny)
            for (int nz = -kReal; nz <= kReal; ++nz) {
                const double v[3] = {d[0] - nx, d[1] - ny, d[2] - nz};
                const double r2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
                const bool origin = (nx == 0 && ny == 0 && nz == 0);
                if (r2 > 9.0 && !origin) continue;  // erfc(2 a) below 2e-17 beyond r = 3
                double w, dw_over_r;  // weight of v and (dw/dr) / r
                if (origin && without_mono) {
                    // (B - 1) / r^3: the point mass's own 1/r^2 removed
                    if (r2 < 1e-12) {
                        // series: B - 1 = -4 a^3 r^3 / (3 sqrt(pi)) + 4 a^5 r^5 / (5 sqrt(pi)) - ...
                        const double a3 = kAlpha * kAlpha * kAlpha;
                        w = -4.0 * a3 / (3.0 * sqrt(kPi)) + 4.0 * a3 * kAlpha * kAlpha * r2 / (5.0 * sqrt(kPi));
                        dw_over_r = 8.0 * a3 * kAlpha * kAlpha / (5.0 * sqrt(kPi));
                    } else {
                        const double r = sqrt(r2);
                        double b, db;
                        ewald_b(r, b, db);
                        // B - 1 without cancellation: -erf(a r) + 2 a r / sqrt(pi) e
                        const double bm1 = -erf(kAlpha * r) + 2.0 * kAlpha * r / sqrt(kPi) *
                                                                  exp(-kAlpha * kAlpha * r2);
                        w = bm1 / (r2 * r);
                        dw_over_r = (db / (r2 * r) - 3.0 * bm1 / (r2 * r2)) / r;
                    }
                } else {
                    if (r2 == 0.0) continue;
                    const double r = sqrt(r2);
                    double b, db;
                    ewald_b(r, b, db);
                    w = b / (r2 * r);
                    dw_over_r = (db / (r2 * r) - 3.0 * b / (r2 * r2)) / r;
                }
                f[0] += v[0] * w;
                f[1] += v[1] * w;
                f[2] += v[2] * w;
                if (jac) {
                    J[0] += w + v[0] * v[0] * dw_over_r;
                    J[1] += v[0] * v[1] * dw_over_r;
                    J[2] += v[0] * v[2] * dw_over_r;
                    J[3] += w + v[1] * v[1] * dw_over_r;
                    J[4] += v[1] * v[2] * dw_over_r;
                    J[5] += w + v[2] * v[2] * dw_over_r;
                }
            }
    for (int mx = -kRecip; mx <= kRecip; ++mx)
        for (int my = -kRecip; my <= kRecip; ++my)
            for (int mz = -kRecip; mz <= kRecip; ++mz) {
                const int m2 = mx * mx + my * my + mz * mz;
                if (m2 == 0 || m2 > 12) continue;  // weights below 1e-14 beyond |m|^2 = 12
                const double k[3] = {2.0 * kPi * mx, 2.0 * kPi * my, 2.0 * kPi * mz};
                const double k2 = k[0] * k[0] + k[1] * k[1] + k[2] * k[2];
                const double wk = 4.0 * kPi * exp(-k2 / (4.0 * kAlpha * kAlpha)) / k2;
                double s, c;
                sincos(k[0] * d[0] + k[1] * d[1] + k[2] * d[2], &s, &c);
                f[0] += k[0] * wk * s;
                f[1] += k[1] * wk * s;
                f[2] += k[2] * wk * s;
                if (jac) {
                    J[0] += k[0] * k[0] * wk * c;
                    J[1] += k[0] * k[1] * wk * c;
                    J[2] += k[0] * k[2] * wk * c;
                    J[3] += k[1] * k[1] * wk * c;
                    J[4] += k[1] * k[2] * wk * c;
                    J[5] += k[2] * k[2] * wk * c;
                }
            }
    if (jac)
        for (int q = 0; q < 6; ++q) jac[q] = J[q];
}

// Grid point (i, j, k) of the octant, spacing 1 / (2 nt): g, its Jacobian
// and its second derivatives H_ijk = d^2 g_i / d_j d_k (symmetric in all
// three indices, g being the gradient of a potential), six float4:
//   (gx, gy, gz, 0 | Jxx, Jxy, Jxz, Jyy | Jyz, Jzz, 0, 0 |
//    Hxxx, Hxxy, Hxxz, Hxyy | Hxyz, Hxzz, Hyyy, Hyyz | Hyzz, Hzzz, 0, 0).
// H by central differences of the analytic Jacobian (step 1e-4, float64).
__global__ void __launch_bounds__(128) k_ewald_table(float4 *table, int nt) {
    const int64_t pts = (int64_t)(nt + 1) * (nt + 1) * (nt + 1);
    const double h = 0.5 / nt;
    const double lin = 4.0 * kPi / 3.0;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < pts;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(t / ((int64_t)(nt + 1) * (nt + 1)));
        const int j = (int)((t / (nt + 1)) % (nt + 1));
        const int k = (int)(t % (nt + 1));
        const double d[3] = {i * h, j * h, k * h};
        double f[3], J[6];
        ewald_force(d, true, f, J);
        // dJ/dd_k: the diagonal (linear) term drops out of the differences
        constexpr double kStep = 1e-4;
        double dJ[3][6];
        for (int k2 = 0; k2 < 3; ++k2) {
            double dp[3] = {d[0], d[1], d[2]}, dm[3] = {d[0], d[1], d[2]};
            dp[k2] += kStep;
            dm[k2] -= kStep;
            double fp[3], fm[3], Jp[6], Jm[6];
            ewald_force(dp, true, fp, Jp);
            ewald_force(dm, true, fm, Jm);
            for (int q = 0; q < 6; ++q) dJ[k2][q] = (Jp[q] - Jm[q]) / (2.0 * kStep);
        }
        // J index: xx 0, xy 1, xz 2, yy 3, yz 4, zz 5; H_ijk = dJ_ij / dd_k
        const double Hxxx = dJ[0][0], Hxxy = dJ[1][0], Hxxz = dJ[2][0], Hxyy = dJ[1][1];
        const double Hxyz = dJ[2][1], Hxzz = dJ[2][2], Hyyy = dJ[1][3], Hyyz = dJ[2][3];
        const double Hyzz = dJ[2][4], Hzzz = dJ[2][5];
        float4 *row = table + 6 * t;
        // g = f_per - mono + (4 pi / 3) d; its Jacobian gains (4 pi / 3) I
        row[0] = make_float4((float)(f[0] + lin * d[0]), (float)(f[1] + lin * d[1]),
                             (float)(f[2] + lin * d[2]), 0.f);
        row[1] = make_float4((float)(J[0] + lin), (float)J[1], (float)J[2], (float)(J[3] + lin));
        row[2] = make_float4((float)J[4], (float)(J[5] + lin), 0.f, 0.f);
        row[3] = make_float4((float)Hxxx, (float)Hxxy, (float)Hxxz, (float)Hxyy);
        row[4] = make_float4((float)Hxyz, (float)Hxzz, (float)Hyyy, (float)Hyyz);
        row[5] = make_float4((float)Hyzz, (float)Hzzz, 0.f, 0.f);
    }
}

// Float64 periodic direct sum: per pair the softened monopole at the
// minimum image (the reference's d^2 > 1e-7 cut) plus f_per - d/|d|^3 of
// that image, the Ewald sums carried to float64 precision.  One block per target.
__global__ void __launch_bounds__(256) k_direct_sum_ewald(const float *__restrict__ px,
                                                          const float *__restrict__ py,
                                                          const float *__restrict__ pz,
                                                          const float *__restrict__ mass,
                                                          int64_t n,
                                                          const int64_t *__restrict__ targets,
                                                          double G, double soft2, double *out) {
    __shared__ double red[3][256];
    const int64_t ti = targets[blockIdx.x];
    const double xi = px[ti], yi = py[ti], zi = pz[ti];
    double ax = 0, ay = 0, az = 0;
    for (int64_t j = threadIdx.x; j < n; j += blockDim.x) {
        double d[3] = {(double)px[j] - xi, (double)py[j] - yi, (double)pz[j] - zi};
        for (int q = 0; q < 3; ++q) d[q] -= rint(d[q]);
        const double d2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
        if (!(d2 > 1e-7)) continue;
        const double m = mass[j];
        const double inv = 1.0 / sqrt(d2 + soft2);
        const double w = m * inv * inv * inv;
        double f[3];
        ewald_force(d, true, f, nullptr);
        ax += w * d[0] + m * f[0];
        ay += w * d[1] + m * f[1];
        az += w * d[2] + m * f[2];
    }
    red[0][threadIdx.x] = ax;
    red[1][threadIdx.x] = ay;
    red[2][threadIdx.x] = az;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s)
            for (int q = 0; q < 3; ++q) red[q][threadIdx.x] += red[q][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int q = 0; q < 3; ++q) out[3 * blockIdx.x + q] = G * red[q][0];
}

}  // namespace cnb

using namespace cnb;

extern "C" int cnb_ewald_table(float *table, int nt, void *stream) {
    if (!table || nt < 2 || nt > 512) return CNB_E_INVALID_ARG;
    if (reinterpret_cast<uintptr_t>(table) & 15) return CNB_E_INVALID_ARG;
    const int64_t pts = (int64_t)(nt + 1) * (nt + 1) * (nt + 1);
    k_ewald_table<<<grid_for(pts, 128), 128, 0, as_stream(stream)>>>(
        reinterpret_cast<float4 *>(table), nt);
    return launch_status();
}

extern "C" int cnb_direct_sum_ewald_f64(const float *px, const float *py, const float *pz,
                                        const float *mass, int64_t n, const int64_t *targets,
                                        int64_t n_targets, double G, double soft, double *out,
                                        void *stream) {
    if (n < 0 || n_targets < 0) return CNB_E_INVALID_ARG;
    if (n_targets == 0) return CNB_OK;
    if (!px || !py || !pz || !mass || !targets || !out) return CNB_E_INVALID_ARG;
    if (n_targets > INT32_MAX) return CNB_E_TOO_LARGE;
    k_direct_sum_ewald<<<(unsigned)n_targets, 256, 0, as_stream(stream)>>>(
        px, py, pz, mass, n, targets, G, soft * soft, out);
    return launch_status();
}
