// controller.cu -- learned opening-angle controller (no reference
// counterpart): bucket features, the fused feature + MLP inference kernel,
// and the training kernels (forward/backward, parameter gradients, Adam).
//
// Network: 12 inputs -> 64 -> 64 -> 1, SiLU hidden activations, output
// theta = THETA_LO + (THETA_HI - THETA_LO) * sigmoid(z), i.e. clipped to
// [0.2, 1.0].  Parameters (CNB_MLP_PARAMS floats, this order):
//   W1[64][12], b1[64], W2[64][64], b2[64], w3[64], b3.
// Inference keeps the weights in bfloat16 and accumulates in float32: the
// first layer in float32 per bucket, the 64 x 64 second layer on the tensor
// cores (mma.sync m16n8k16, its input -- the first layer's SiLU outputs --
// rounded to bfloat16); training keeps float32 master weights.
//
// Features of a bucket (its subtree node v, ancestors p1..p3), lengths in
// units of the box's mean body spacing s = (body mass)^(1/3):
//   f0  log2(extent(v) / s)
//   f1  log2(mean |a| of the bucket's bodies at the previous step over
//       G mass(p3) / extent(p3)^2, the force scale of the third ancestor)
//       / 4: the relative force error a given theta leaves grows as the
//       bucket's own acceleration shrinks
//   f2  log2(density(v) / mean density)
//   f3+3k..f5+3k (k = 0..2, ancestor p_{k+1}):
//       log2(extent(p) / extent(v)), log2(mass(p) / mass(v)),
//       |com(p) - com(v)| / extent(p)
#include <cuda_bf16.h>

#include "common.cuh"

namespace cnb {

constexpr int kIn = 12, kH = 64;
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kH * kIn, kOffW2 = kOffB1 + kH,
              kOffB2 = kOffW2 + kH * kH, kOffW3 = kOffB2 + kH, kOffB3 = kOffW3 + kH;
constexpr int kParams = kOffB3 + 1;  // 5057
constexpr float kThetaLo = 0.2f, kThetaHi = 1.0f;
static_assert(kParams == CNB_MLP_PARAMS, "parameter count");

__device__ __forceinline__ float sigmoidf_(float x) { return 1.f / (1.f + __expf(-x)); }
__device__ __forceinline__ float siluf_(float x) { return x * sigmoidf_(x); }

__device__ __forceinline__ float node_extent(const float4 *aabb, int v) {
    const float4 lo = aabb[2 * v], hi = aabb[2 * v + 1];
    return fmaxf(hi.x - lo.x, fmaxf(hi.y - lo.y, hi.z - lo.z));
}

// Mean |a| of a bucket's bodies (previous step; row perm[i] of accel for
// sorted body i), by one thread.
__device__ float bucket_mean_accel(const float *__restrict__ accel, const uint32_t *__restrict__ perm,
                                   int4 bk) {
    float amean = 0.f;
    for (int k = 0; k < bk.y; ++k) {
        const int64_t i = (int64_t)bk.x + k;
        const int64_t r = perm ? (int64_t)perm[i] : i;
        const float ax = accel[3 * r], ay = accel[3 * r + 1], az = accel[3 * r + 2];
        amean += sqrtf(ax * ax + ay * ay + az * az);
    }
    return amean / (float)bk.y;
}

__device__ void bucket_features(const float4 *__restrict__ rec, const float4 *__restrict__ aabb,
                                const int32_t *__restrict__ parents, float amean, int4 bk,
                                float f[kIn]) {
    const int v = bk.z;
    const float4 A = rec[2 * v];
    const float m_body = A.w / (float)bk.y;
    const float s = cbrtf(fmaxf(m_body, 1e-30f));  // mean spacing of the box (unit cube)
    const float4 lo = aabb[2 * v], hi = aabb[2 * v + 1];
    const float ext = fmaxf(node_extent(aabb, v), 1e-3f * s);
    const float vol = (hi.x - lo.x + s) * (hi.y - lo.y + s) * (hi.z - lo.z + s);
    f[0] = __log2f(ext / s);
    f[2] = __log2f((float)bk.y * s * s * s / vol);
    int p = v;
    float pe = ext, pm = A.w;
    for (int k = 0; k < 3; ++k) {
        const int q = parents[p];
        if (q >= 0) p = q;
        const float4 P = rec[2 * p];
        pe = fmaxf(node_extent(aabb, p), ext);
        pm = fmaxf(P.w, A.w);
        const float dx = P.x - A.x, dy = P.y - A.y, dz = P.z - A.z;
        f[3 + 3 * k] = __log2f(pe / ext);
        f[4 + 3 * k] = __log2f(pm / A.w);
        f[5 + 3 * k] = sqrtf(dx * dx + dy * dy + dz * dz) / pe;
    }
    // G = 1 in the box's units: the scale is the third ancestor's M / l^2
    f[1] = 0.25f * __log2f(fmaxf(amean * pe * pe / pm, 1e-6f));
}

__global__ void __launch_bounds__(256) k_features(const float4 *__restrict__ rec,
                                                  const float4 *__restrict__ aabb,
                                                  const int32_t *__restrict__ parents,
                                                  const int32_t *__restrict__ ws,
                                                  const float *__restrict__ accel,
                                                  const uint32_t *__restrict__ perm,
                                                  float *__restrict__ out, int max_buckets) {
    const int nb = min(ws[0], max_buckets);
    const int4 *buckets = reinterpret_cast<const int4 *>(ws + 4);
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < nb; g += gridDim.x * blockDim.x) {
        float f[kIn];
        const int4 bk = buckets[g];
        bucket_features(rec, aabb, parents, bucket_mean_accel(accel, perm, bk), bk, f);
#pragma unroll
        for (int k = 0; k < kIn; ++k) out[(int64_t)g * kIn + k] = f[k];
    }
}

// z = network output before the output squashing, float32 weights in
// shared memory.  Hidden unit j of layer 1 is formed once and scattered into
// the 64 layer-2 accumulators, so only those stay in registers.
__device__ __forceinline__ float mlp_forward(const float *__restrict__ w, const float x[kIn]) {
    float a2[kH];
#pragma unroll
    for (int k = 0; k < kH; ++k) a2[k] = w[kOffB2 + k];
#pragma unroll 1
    for (int j = 0; j < kH; ++j) {
        float a = w[kOffB1 + j];
#pragma unroll
        for (int i = 0; i < kIn; ++i) a = fmaf(w[kOffW1 + j * kIn + i], x[i], a);
        const float h = siluf_(a);
#pragma unroll
        for (int k = 0; k < kH; ++k) a2[k] = fmaf(w[kOffW2 + k * kH + j], h, a2[k]);
    }
    float z = w[kOffB3];
#pragma unroll
    for (int k = 0; k < kH; ++k) z = fmaf(w[kOffW3 + k], siluf_(a2[k]), z);
    return z;
}

__device__ __forceinline__ float theta_of(float z) {
    return kThetaLo + (kThetaHi - kThetaLo) * sigmoidf_(z);
}

// Fused inference with the 64 x 64 hidden layer on the tensor cores: one
// warp takes 32 buckets (two 16-row tiles).  Each lane forms one bucket's
// features and its first layer in float32 (12 -> 64, SiLU) and stores the
// hidden vector as bfloat16 in shared memory; the second layer is
// mma.sync.m16n8k16 (bf16 inputs, float32 accumulation) against W2 in
// bfloat16; bias, SiLU and the output layer are applied on the accumulator
// fragments and summed over the four lanes that share a row.
constexpr int kMmaWarps = 4;
constexpr int kHPad = kH + 8;  // bf16 per row of the hidden tiles: staggers the banks

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t *>(&v);
}

__device__ __forceinline__ void mma_bf16_16816(float (&d)[4], const uint32_t (&a)[4],
                                               const uint32_t (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
        "{%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, {%0, %1, %2, %3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__global__ void __launch_bounds__(kMmaWarps * 32) k_controller_mma(
    const float4 *__restrict__ rec, const float4 *__restrict__ aabb,
    const int32_t *__restrict__ parents, const int32_t *__restrict__ ws,
    const float *__restrict__ accel, const uint32_t *__restrict__ perm,
    const __nv_bfloat16 *__restrict__ wbf, float *__restrict__ theta, int max_buckets) {
    // float32: W1, b1, b2, w3, b3; bfloat16: W2 rows (output unit) of kHPad
    __shared__ float w1[kH * kIn], b1[kH], b2[kH], w3[kH];
    __shared__ float b3;
    __shared__ __align__(16) __nv_bfloat16 w2[kH * kHPad];
    __shared__ __align__(16) __nv_bfloat16 hid[kMmaWarps][32 * kHPad];
    for (int i = threadIdx.x; i < kH * kIn; i += blockDim.x) w1[i] = __bfloat162float(wbf[kOffW1 + i]);
    for (int i = threadIdx.x; i < kH; i += blockDim.x) {
        b1[i] = __bfloat162float(wbf[kOffB1 + i]);
        b2[i] = __bfloat162float(wbf[kOffB2 + i]);
        w3[i] = __bfloat162float(wbf[kOffW3 + i]);
    }
    for (int i = threadIdx.x; i < kH * kH; i += blockDim.x) w2[(i / kH) * kHPad + i % kH] = wbf[kOffW2 + i];
    if (threadIdx.x == 0) b3 = __bfloat162float(wbf[kOffB3]);
    __syncthreads();
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int gid = lane >> 2, tig = lane & 3;
    const int nb = min(ws[0], max_buckets);
    const int4 *buckets = reinterpret_cast<const int4 *>(ws + 4);
    __nv_bfloat16 *h = hid[wib];
    for (int base = (blockIdx.x * kMmaWarps + wib) * 32; base < nb; base += gridDim.x * kMmaWarps * 32) {
        // one bucket per lane: features and the first layer in float32
        const int g = base + lane;
        if (g < nb) {
            const int4 bk = buckets[g];
            float f[kIn];
            bucket_features(rec, aabb, parents, bucket_mean_accel(accel, perm, bk), bk, f);
#pragma unroll 4
            for (int j = 0; j < kH; j += 2) {
                float a0 = b1[j], a1 = b1[j + 1];
#pragma unroll
                for (int i = 0; i < kIn; ++i) {
                    a0 = fmaf(w1[j * kIn + i], f[i], a0);
                    a1 = fmaf(w1[(j + 1) * kIn + i], f[i], a1);
                }
                *reinterpret_cast<uint32_t *>(h + lane * kHPad + j) = pack_bf16(siluf_(a0), siluf_(a1));
            }
        } else {
            for (int j = 0; j < kH; j += 2) *reinterpret_cast<uint32_t *>(h + lane * kHPad + j) = 0u;
        }
        __syncwarp();
        // second layer: rows = buckets, columns = hidden units, k = first-layer units
        float z[2][2] = {{0.f, 0.f}, {0.f, 0.f}};  // [m tile][row gid / gid + 8]
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
            uint32_t a[4][4];
            const __nv_bfloat16 *r0 = h + (mt * 16 + gid) * kHPad, *r1 = r0 + 8 * kHPad;
#pragma unroll
            for (int kt = 0; kt < 4; ++kt) {
                const int c = kt * 16 + tig * 2;
                a[kt][0] = *reinterpret_cast<const uint32_t *>(r0 + c);
                a[kt][1] = *reinterpret_cast<const uint32_t *>(r1 + c);
                a[kt][2] = *reinterpret_cast<const uint32_t *>(r0 + c + 8);
                a[kt][3] = *reinterpret_cast<const uint32_t *>(r1 + c + 8);
            }
#pragma unroll
            for (int nt = 0; nt < kH / 8; ++nt) {
                float d[4] = {0.f, 0.f, 0.f, 0.f};
                const __nv_bfloat16 *wr = w2 + (nt * 8 + gid) * kHPad;  // output unit nt*8 + gid
#pragma unroll
                for (int kt = 0; kt < 4; ++kt) {
                    const int c = kt * 16 + tig * 2;
                    const uint32_t b[2] = {*reinterpret_cast<const uint32_t *>(wr + c),
                                           *reinterpret_cast<const uint32_t *>(wr + c + 8)};
                    mma_bf16_16816(d, a[kt], b);
                }
                const int col = nt * 8 + tig * 2;
                z[mt][0] = fmaf(w3[col], siluf_(d[0] + b2[col]), z[mt][0]);
                z[mt][0] = fmaf(w3[col + 1], siluf_(d[1] + b2[col + 1]), z[mt][0]);
                z[mt][1] = fmaf(w3[col], siluf_(d[2] + b2[col]), z[mt][1]);
                z[mt][1] = fmaf(w3[col + 1], siluf_(d[3] + b2[col + 1]), z[mt][1]);
            }
        }
        // the four lanes of a row group hold its partial sums
#pragma unroll
        for (int mt = 0; mt < 2; ++mt)
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                z[mt][q] += __shfl_xor_sync(0xffffffffu, z[mt][q], 1);
                z[mt][q] += __shfl_xor_sync(0xffffffffu, z[mt][q], 2);
            }
        if (tig == 0) {
#pragma unroll
            for (int mt = 0; mt < 2; ++mt)
#pragma unroll
                for (int q = 0; q < 2; ++q) {
                    const int gg = base + mt * 16 + gid + 8 * q;
                    if (gg < nb) theta[gg] = theta_of(z[mt][q] + b3);
                }
        }
        __syncwarp();
    }
}

// Inference on given features with float32 weights (training evaluation).
__global__ void __launch_bounds__(256) k_mlp_predict(const float *__restrict__ x, int n,
                                                     const float *__restrict__ wg,
                                                     float *__restrict__ theta) {
    __shared__ float w[kParams];
    for (int i = threadIdx.x; i < kParams; i += blockDim.x) w[i] = wg[i];
    __syncthreads();
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        float f[kIn];
#pragma unroll
        for (int i = 0; i < kIn; ++i) f[i] = x[(int64_t)s * kIn + i];
        theta[s] = theta_of(mlp_forward(w, f));
    }
}

// Training, phase 1 (one thread per sample): forward pass and the backward
// pass down to the pre-activation gradients.  Loss per sample:
//   L = c * (theta - y)^2,  c = over_weight if theta > y else 1,
// averaged over the n samples (over-estimating theta costs accuracy, so it
// can be weighted up).  Writes H1, DA1, H2, DA2 ([n, 64] each), DZ [n] and
// adds the loss sum into *loss.
__global__ void __launch_bounds__(128) k_mlp_backward_acts(
    const float *__restrict__ x, const float *__restrict__ y, int n, const float *__restrict__ wg,
    float over_weight, float *__restrict__ H1, float *__restrict__ DA1, float *__restrict__ H2,
    float *__restrict__ DA2, float *__restrict__ DZ, float *__restrict__ loss) {
    __shared__ float w[kParams];
    for (int i = threadIdx.x; i < kParams; i += blockDim.x) w[i] = wg[i];
    __syncthreads();
    float lsum = 0.f;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        float f[kIn];
#pragma unroll
        for (int i = 0; i < kIn; ++i) f[i] = x[(int64_t)s * kIn + i];
        float* h1row = H1 + (int64_t)s * kH;
        float* da1row = DA1 + (int64_t)s * kH;
        float a2[kH];
#pragma unroll
        for (int k = 0; k < kH; ++k) a2[k] = w[kOffB2 + k];
#pragma unroll 1
        for (int j = 0; j < kH; ++j) {
            float a = w[kOffB1 + j];
#pragma unroll
            for (int i = 0; i < kIn; ++i) a = fmaf(w[kOffW1 + j * kIn + i], f[i], a);
            const float h = siluf_(a);
            h1row[j] = h;
            da1row[j] = a;  // layer-1 pre-activation, turned into its gradient below
#pragma unroll
            for (int k = 0; k < kH; ++k) a2[k] = fmaf(w[kOffW2 + k * kH + j], h, a2[k]);
        }
        float z = w[kOffB3];
#pragma unroll
        for (int k = 0; k < kH; ++k) {
            const float h = siluf_(a2[k]);
            H2[(int64_t)s * kH + k] = h;
            z = fmaf(w[kOffW3 + k], h, z);
        }
        const float sg = sigmoidf_(z);
        const float th = kThetaLo + (kThetaHi - kThetaLo) * sg;
        const float diff = th - y[s];
        const float c = diff > 0.f ? over_weight : 1.f;
        lsum += c * diff * diff;
        const float dz = (2.f * c * diff / (float)n) * (kThetaHi - kThetaLo) * sg * (1.f - sg);
        DZ[s] = dz;
#pragma unroll
        for (int k = 0; k < kH; ++k) {
            const float sa = sigmoidf_(a2[k]);
            a2[k] = dz * w[kOffW3 + k] * sa * (1.f + a2[k] * (1.f - sa));  // now dL/da2
            DA2[(int64_t)s * kH + k] = a2[k];
        }
#pragma unroll 1
        for (int j = 0; j < kH; ++j) {
            float dh = 0.f;
#pragma unroll
            for (int k = 0; k < kH; ++k) dh = fmaf(w[kOffW2 + k * kH + j], a2[k], dh);
            const float a = da1row[j];
            const float sa = sigmoidf_(a);
            da1row[j] = dh * sa * (1.f + a * (1.f - sa));
        }
    }
    for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, lsum / (float)n);
}

// Training, phase 2: parameter gradients as sums over samples.  Block r < 64
// computes row r of W1 (12 inputs) and b1; block 64 + r row r of W2 and b2;
// block 128 computes w3 and b3.  Threads stride over samples; each output
// is reduced in shared memory.  grad must hold CNB_MLP_PARAMS floats.
__global__ void __launch_bounds__(256) k_mlp_param_grads(
    const float *__restrict__ x, int n, const float *__restrict__ H1, const float *__restrict__ DA1,
    const float *__restrict__ H2, const float *__restrict__ DA2, const float *__restrict__ DZ,
    float *__restrict__ grad) {
    __shared__ float red[kH + 1][8];
    const int r = blockIdx.x;
    float acc[kH + 1];
#pragma unroll
    for (int k = 0; k <= kH; ++k) acc[k] = 0.f;
    int cols = 0;
    const float *rowsrc = nullptr;  // per-sample scalar multiplier (column r)
    const float *insrc = nullptr;   // per-sample input vector
    int in_stride = 0;
    if (r < kH) {
        cols = kIn; rowsrc = DA1; insrc = x; in_stride = kIn;
    } else if (r < 2 * kH) {
        cols = kH; rowsrc = DA2; insrc = H1; in_stride = kH;
    } else {
        cols = kH; rowsrc = DZ; insrc = H2; in_stride = kH;
    }
    const int rr = r < 2 * kH ? (r % kH) : 0;
    for (int s = threadIdx.x; s < n; s += blockDim.x) {
        const float d = (r < 2 * kH) ? rowsrc[(int64_t)s * kH + rr] : rowsrc[s];
#pragma unroll
        for (int k = 0; k < kH; ++k)
            if (k < cols) acc[k] = fmaf(d, insrc[(int64_t)s * in_stride + k], acc[k]);
        acc[kH] += d;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k <= kH; ++k) {
        float v = acc[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) red[k][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x <= kH) {
        const int k = threadIdx.x;
        if (k < cols || k == kH) {
            float v = 0.f;
            for (int w8 = 0; w8 < (int)(blockDim.x >> 5); ++w8) v += red[k][w8];
            if (r < kH) {
                if (k < kH) grad[kOffW1 + rr * kIn + k] = v; else grad[kOffB1 + rr] = v;
            } else if (r < 2 * kH) {
                if (k < kH) grad[kOffW2 + rr * kH + k] = v; else grad[kOffB2 + rr] = v;
            } else {
                if (k < kH) grad[kOffW3 + k] = v; else grad[kOffB3] = v;
            }
        }
    }
}

__global__ void k_adam(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                       float *__restrict__ v, int n, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

__global__ void k_to_bf16(const float *__restrict__ src, __nv_bfloat16 *__restrict__ dst, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        dst[i] = __float2bfloat16_rn(src[i]);
}

}  // namespace cnb

using namespace cnb;

extern "C" int cnb_bucket_features(const float *node_table, const int32_t *parents,
                                   const int32_t *workspace, int64_t n, const float *accel,
                                   const uint32_t *perm, float *features, int max_buckets,
                                   void *stream) {
    if (n < 1 || !node_table || !parents || !workspace || !accel || !features || max_buckets < 0)
        return CNB_E_INVALID_ARG;
    const int64_t m = 2 * n - 1;
    const float4 *rec = reinterpret_cast<const float4 *>(node_table);
    k_features<<<grid_for(max_buckets, 256), 256, 0, as_stream(stream)>>>(
        rec, rec + 2 * m, parents, workspace, accel, perm, features, max_buckets);
    return launch_status();
}

extern "C" int cnb_controller_theta(const float *node_table, const int32_t *parents,
                                    const int32_t *workspace, int64_t n, const float *accel,
                                    const uint32_t *perm, const void *weights_bf16, float *theta,
                                    int max_buckets, void *stream) {
    if (n < 1 || !node_table || !parents || !workspace || !accel || !weights_bf16 || !theta ||
        max_buckets < 0)
        return CNB_E_INVALID_ARG;
    const int64_t m = 2 * n - 1;
    const float4 *rec = reinterpret_cast<const float4 *>(node_table);
    k_controller_mma<<<grid_for(max_buckets, kMmaWarps * 32, 148 * 4), kMmaWarps * 32, 0,
                       as_stream(stream)>>>(rec, rec + 2 * m, parents, workspace, accel, perm,
                                            reinterpret_cast<const __nv_bfloat16 *>(weights_bf16),
                                            theta, max_buckets);
    return launch_status();
}

extern "C" int cnb_mlp_predict(const float *features, int n, const float *weights, float *theta,
                               void *stream) {
    if (n < 0 || (n > 0 && (!features || !weights || !theta))) return CNB_E_INVALID_ARG;
    if (n == 0) return CNB_OK;
    k_mlp_predict<<<grid_for(n, 256, 148 * 4), 256, 0, as_stream(stream)>>>(features, n, weights,
                                                                            theta);
    return launch_status();
}

extern "C" int cnb_mlp_grad(const float *features, const float *labels, int n,
                            const float *weights, float over_weight, float *scratch,
                            float *grad, float *loss, void *stream) {
    if (n < 1 || !features || !labels || !weights || !scratch || !grad || !loss)
        return CNB_E_INVALID_ARG;
    cudaStream_t st = as_stream(stream);
    float *H1 = scratch, *DA1 = H1 + (int64_t)n * kH, *H2 = DA1 + (int64_t)n * kH,
          *DA2 = H2 + (int64_t)n * kH, *DZ = DA2 + (int64_t)n * kH;
    CNB_CUDA(cudaMemsetAsync(loss, 0, sizeof(float), st));
    k_mlp_backward_acts<<<grid_for(n, 128, 148 * 8), 128, 0, st>>>(
        features, labels, n, weights, over_weight, H1, DA1, H2, DA2, DZ, loss);
    CNB_TRY(launch_status());
    k_mlp_param_grads<<<2 * kH + 1, 256, 0, st>>>(features, n, H1, DA1, H2, DA2, DZ, grad);
    return launch_status();
}

extern "C" int cnb_adam_step(float *params, const float *grad, float *m, float *v, int n,
                             float lr, float beta1, float beta2, float eps, int t, void *stream) {
    if (n < 1 || !params || !grad || !m || !v || t < 1) return CNB_E_INVALID_ARG;
    const float c1 = 1.f - powf(beta1, (float)t), c2 = 1.f - powf(beta2, (float)t);
    k_adam<<<grid_for(n, 256), 256, 0, as_stream(stream)>>>(params, grad, m, v, n, lr, beta1,
                                                           beta2, eps, c1, c2);
    return launch_status();
}

extern "C" int cnb_to_bf16(const float *src, void *dst, int n, void *stream) {
    if (n < 0 || (n > 0 && (!src || !dst))) return CNB_E_INVALID_ARG;
    if (n == 0) return CNB_OK;
    k_to_bf16<<<grid_for(n, 256), 256, 0, as_stream(stream)>>>(
        src, reinterpret_cast<__nv_bfloat16 *>(dst), n);
    return launch_status();
}
