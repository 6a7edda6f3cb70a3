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

// ---------------------------------------------------------------- training on the tensor cores
// The same loss and gradients with the three 64-wide contractions on the
// tensor cores (mma.sync m16n8k16, bfloat16 operands, float32 accumulation):
// the forward second layer A2 = H1 W2^T, the backward dH1 = dA2 W2, and the
// parameter gradients dW2 = dA2^T H1 and dW1 = dA1^T X summed over the
// samples.  Layer 1's pre-activations, SiLU and its derivative, the loss,
// dz, the bias sums and dw3 stay in float32.
//
// k_mlp_train_mma: one warp per 32 samples.  Lane s forms sample s's first
// layer in float32 and stores H1 in bfloat16 (shared, row-major, and
// transposed to global for the parameter GEMM); the warp runs A2 on the
// tensor cores, finishes the forward pass and the loss on the accumulator
// fragments, forms dA2 there, runs dH1 = dA2 W2 on the tensor cores and
// forms dA1 (layer 1 recomputed from the staged inputs, the same fmaf
// order as the forward pass).  dA2, dA1 and X go to global memory
// transposed ([unit][sample], bfloat16, samples padded to a multiple of 32
// with zero gradients).  Bias sums, dw3 and the loss are reduced in
// registers and added once per warp.
constexpr int kTW = 4;              // warps per block
constexpr int kTPad = kH + 8;       // bfloat16 per row of the activation tiles
constexpr int kTWeightBytes = (kH * kIn + 3 * kH + 4) * 4;             // w1, b1, b2, w3, b3
constexpr int kTWarpBytes = 32 * kIn * 4 + 2 * 32 * kTPad * 2;         // inputs, H1, dA tiles
constexpr int kTSmem = kTWeightBytes + 2 * kH * kTPad * 2 + kTW * kTWarpBytes;
static_assert(kTWeightBytes % 16 == 0 && kTWarpBytes % 16 == 0, "16-byte aligned regions");

__device__ __forceinline__ uint32_t ld_u32(const __nv_bfloat16 *p) {
    return *reinterpret_cast<const uint32_t *>(p);
}

__global__ void __launch_bounds__(kTW * 32) k_mlp_train_mma(
    const float *__restrict__ x, const float *__restrict__ y, int n, int n32,
    const float *__restrict__ wg, float over_weight, __nv_bfloat16 *__restrict__ XT,
    __nv_bfloat16 *__restrict__ H1T, __nv_bfloat16 *__restrict__ DA2T,
    __nv_bfloat16 *__restrict__ DA1T, float *__restrict__ grad, float *__restrict__ loss) {
    extern __shared__ __align__(16) unsigned char t_smem[];
    float *w1 = reinterpret_cast<float *>(t_smem);
    float *b1 = w1 + kH * kIn, *b2 = b1 + kH, *w3 = b2 + kH, *b3p = w3 + kH;
    __nv_bfloat16 *w2 = reinterpret_cast<__nv_bfloat16 *>(t_smem + kTWeightBytes);  // [k][j]
    __nv_bfloat16 *w2t = w2 + kH * kTPad;                                            // [j][k]
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int gid = lane >> 2, tig = lane & 3;
    unsigned char *wbase = reinterpret_cast<unsigned char *>(w2t + kH * kTPad) + wib * kTWarpBytes;
    float *sx = reinterpret_cast<float *>(wbase);                                 // [32][12]
    __nv_bfloat16 *hid = reinterpret_cast<__nv_bfloat16 *>(wbase + 32 * kIn * 4);  // [32][kTPad]
    __nv_bfloat16 *dbuf = hid + 32 * kTPad;                                       // [32][kTPad]
    for (int i = threadIdx.x; i < kH * kIn; i += blockDim.x) w1[i] = wg[kOffW1 + i];
    for (int i = threadIdx.x; i < kH; i += blockDim.x) {
        b1[i] = wg[kOffB1 + i];
        b2[i] = wg[kOffB2 + i];
        w3[i] = wg[kOffW3 + i];
    }
    if (threadIdx.x == 0) b3p[0] = wg[kOffB3];
    for (int i = threadIdx.x; i < kH * kH; i += blockDim.x) {
        const int k = i / kH, j = i % kH;
        const __nv_bfloat16 v = __float2bfloat16_rn(wg[kOffW2 + i]);
        w2[k * kTPad + j] = v;
        w2t[j * kTPad + k] = v;
    }
    __syncthreads();
    const float b3 = b3p[0];
    float acc_b1[16], acc_b2[16], acc_w3[16];  // column nt * 8 + tig * 2 + e at index 2 nt + e
#pragma unroll
    for (int c = 0; c < 16; ++c) acc_b1[c] = acc_b2[c] = acc_w3[c] = 0.f;
    float acc_b3 = 0.f, lsum = 0.f;
    for (int base = (blockIdx.x * kTW + wib) * 32; base < n32; base += gridDim.x * kTW * 32) {
        const int s = base + lane;
        // layer 1, one sample per lane, float32
        float xv[kIn];
#pragma unroll
        for (int i = 0; i < kIn; ++i) {
            xv[i] = s < n ? x[(int64_t)s * kIn + i] : 0.f;
            sx[lane * kIn + i] = xv[i];
        }
#pragma unroll
        for (int i = 0; i < 16; ++i) XT[(int64_t)i * n32 + s] = __float2bfloat16_rn(i < kIn ? xv[i] : 0.f);
#pragma unroll 4
        for (int j = 0; j < kH; j += 2) {
            float a0 = b1[j], a1 = b1[j + 1];
#pragma unroll
            for (int i = 0; i < kIn; ++i) {
                a0 = fmaf(w1[j * kIn + i], xv[i], a0);
                a1 = fmaf(w1[(j + 1) * kIn + i], xv[i], a1);
            }
            const __nv_bfloat162 hb = __floats2bfloat162_rn(siluf_(a0), siluf_(a1));
            *reinterpret_cast<__nv_bfloat162 *>(hid + lane * kTPad + j) = hb;
            H1T[(int64_t)j * n32 + s] = hb.x;
            H1T[(int64_t)(j + 1) * n32 + s] = hb.y;
        }
        __syncwarp();
        // per 16-sample row tile: A2 = H1 W2^T on the tensor cores (rows =
        // samples, columns = units), z, the loss, dz and dA2 on the fragments
#pragma unroll 1
        for (int mt = 0; mt < 2; ++mt) {
            float d[8][4];
            {
                uint32_t a[4][4];
                const __nv_bfloat16 *r0 = hid + (mt * 16 + gid) * kTPad, *r1 = r0 + 8 * kTPad;
#pragma unroll
                for (int kt = 0; kt < 4; ++kt) {
                    const int c = kt * 16 + tig * 2;
                    a[kt][0] = ld_u32(r0 + c);
                    a[kt][1] = ld_u32(r1 + c);
                    a[kt][2] = ld_u32(r0 + c + 8);
                    a[kt][3] = ld_u32(r1 + c + 8);
                }
#pragma unroll
                for (int nt = 0; nt < 8; ++nt) {
                    d[nt][0] = d[nt][1] = d[nt][2] = d[nt][3] = 0.f;
                    const __nv_bfloat16 *wr = w2 + (nt * 8 + gid) * kTPad;
#pragma unroll
                    for (int kt = 0; kt < 4; ++kt) {
                        const int c = kt * 16 + tig * 2;
                        const uint32_t b[2] = {ld_u32(wr + c), ld_u32(wr + c + 8)};
                        mma_bf16_16816(d[nt], a[kt], b);
                    }
                }
            }
            // z per sample: the four lanes of a row group hold its partial sums
            float zp[2] = {0.f, 0.f};
#pragma unroll
            for (int nt = 0; nt < 8; ++nt)
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int col = nt * 8 + tig * 2 + (e & 1);
                    d[nt][e] += b2[col];
                    zp[e >> 1] = fmaf(w3[col], siluf_(d[nt][e]), zp[e >> 1]);
                }
            float dzr[2];
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                float z = zp[q];
                z += __shfl_xor_sync(0xffffffffu, z, 1);
                z += __shfl_xor_sync(0xffffffffu, z, 2);
                z += b3;
                const int sr = base + mt * 16 + gid + 8 * q;
                float dz = 0.f;
                if (sr < n) {
                    const float sg = sigmoidf_(z);
                    const float diff = kThetaLo + (kThetaHi - kThetaLo) * sg - y[sr];
                    const float c = diff > 0.f ? over_weight : 1.f;
                    if (tig == 0) lsum += c * diff * diff;
                    dz = (2.f * c * diff / (float)n) * (kThetaHi - kThetaLo) * sg * (1.f - sg);
                }
                dzr[q] = dz;
                if (tig == 0) acc_b3 += dz;
            }
            // dA2 on the fragments; dw3 and db2 sums
#pragma unroll
            for (int nt = 0; nt < 8; ++nt) {
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int col = nt * 8 + tig * 2 + (e & 1);
                    const float a2 = d[nt][e], dz = dzr[e >> 1];
                    const float sa = sigmoidf_(a2);
                    acc_w3[2 * nt + (e & 1)] = fmaf(dz, a2 * sa, acc_w3[2 * nt + (e & 1)]);
                    d[nt][e] = dz * w3[col] * sa * (1.f + a2 * (1.f - sa));
                    acc_b2[2 * nt + (e & 1)] += d[nt][e];
                }
                const int r = mt * 16 + gid, c = nt * 8 + tig * 2;
                *reinterpret_cast<__nv_bfloat162 *>(dbuf + r * kTPad + c) =
                    __floats2bfloat162_rn(d[nt][0], d[nt][1]);
                *reinterpret_cast<__nv_bfloat162 *>(dbuf + (r + 8) * kTPad + c) =
                    __floats2bfloat162_rn(d[nt][2], d[nt][3]);
            }
        }
        __syncwarp();
        for (int k = 0; k < kH; ++k) DA2T[(int64_t)k * n32 + s] = dbuf[lane * kTPad + k];
        // per row tile: dH1 = dA2 W2 on the tensor cores, then dA1 = dH1 * SiLU'(A1)
        // with A1 recomputed from the staged inputs (the forward pass's fmaf order)
#pragma unroll 1
        for (int mt = 0; mt < 2; ++mt) {
            float d[8][4];
            {
                uint32_t a[4][4];
                const __nv_bfloat16 *r0 = dbuf + (mt * 16 + gid) * kTPad, *r1 = r0 + 8 * kTPad;
#pragma unroll
                for (int kt = 0; kt < 4; ++kt) {
                    const int c = kt * 16 + tig * 2;
                    a[kt][0] = ld_u32(r0 + c);
                    a[kt][1] = ld_u32(r1 + c);
                    a[kt][2] = ld_u32(r0 + c + 8);
                    a[kt][3] = ld_u32(r1 + c + 8);
                }
                __syncwarp();  // this tile's dA2 is read by every lane before dA1 overwrites it
#pragma unroll
                for (int nt = 0; nt < 8; ++nt) {
                    d[nt][0] = d[nt][1] = d[nt][2] = d[nt][3] = 0.f;
                    const __nv_bfloat16 *wr = w2t + (nt * 8 + gid) * kTPad;
#pragma unroll
                    for (int kt = 0; kt < 4; ++kt) {
                        const int c = kt * 16 + tig * 2;
                        const uint32_t b[2] = {ld_u32(wr + c), ld_u32(wr + c + 8)};
                        mma_bf16_16816(d[nt], a[kt], b);
                    }
                }
            }
#pragma unroll
            for (int nt = 0; nt < 8; ++nt) {
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int r = mt * 16 + gid + 8 * (e >> 1), j = nt * 8 + tig * 2 + (e & 1);
                    float a1 = b1[j];
#pragma unroll
                    for (int i = 0; i < kIn; ++i) a1 = fmaf(w1[j * kIn + i], sx[r * kIn + i], a1);
                    const float sa = sigmoidf_(a1);
                    d[nt][e] *= sa * (1.f + a1 * (1.f - sa));
                    acc_b1[2 * nt + (e & 1)] += d[nt][e];
                }
                const int r = mt * 16 + gid, c = nt * 8 + tig * 2;
                *reinterpret_cast<__nv_bfloat162 *>(dbuf + r * kTPad + c) =
                    __floats2bfloat162_rn(d[nt][0], d[nt][1]);
                *reinterpret_cast<__nv_bfloat162 *>(dbuf + (r + 8) * kTPad + c) =
                    __floats2bfloat162_rn(d[nt][2], d[nt][3]);
            }
        }
        __syncwarp();
        for (int j = 0; j < kH; ++j) DA1T[(int64_t)j * n32 + s] = dbuf[lane * kTPad + j];
        __syncwarp();
    }
    // column sums over the eight row groups of the warp, one atomic per column
#pragma unroll
    for (int c = 0; c < 16; ++c) {
        float v1 = acc_b1[c], v2 = acc_b2[c], v3 = acc_w3[c];
#pragma unroll
        for (int o = 4; o < 32; o <<= 1) {
            v1 += __shfl_xor_sync(0xffffffffu, v1, o);
            v2 += __shfl_xor_sync(0xffffffffu, v2, o);
            v3 += __shfl_xor_sync(0xffffffffu, v3, o);
        }
        if (gid == 0) {
            const int col = (c >> 1) * 8 + tig * 2 + (c & 1);
            atomicAdd(grad + kOffB1 + col, v1);
            atomicAdd(grad + kOffB2 + col, v2);
            atomicAdd(grad + kOffW3 + col, v3);
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        acc_b3 += __shfl_xor_sync(0xffffffffu, acc_b3, o);
        lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
    }
    if (lane == 0) {
        atomicAdd(grad + kOffB3, acc_b3);
        atomicAdd(loss, lsum / (float)n);
    }
}

// dW2 = dA2^T H1 (64 x 64) and dW1 = dA1^T X (64 x 12, X padded to 16) over
// the samples of one chunk per block, on the tensor cores.  Warp w takes
// row tile w & 3 of both outputs, column tiles 4 (w >> 2) .. + 3 of dW2 and
// column tile w >> 2 of dW1; both operands are read from the transposed
// [unit][sample] arrays, so every fragment register is two consecutive
// samples.  Partial sums are added into grad.
constexpr int kPW = 8;
__global__ void __launch_bounds__(kPW * 32) k_mlp_param_mma(
    const __nv_bfloat16 *__restrict__ XT, const __nv_bfloat16 *__restrict__ H1T,
    const __nv_bfloat16 *__restrict__ DA2T, const __nv_bfloat16 *__restrict__ DA1T, int n32,
    int chunk, float *__restrict__ grad) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int gid = lane >> 2, tig = lane & 3;
    const int mt = w & 3, nq = w >> 2;
    const int k_begin = blockIdx.x * chunk, k_end = min(n32, k_begin + chunk);
    float c2[4][4], c1[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int q = 0; q < 4; ++q) c2[q][0] = c2[q][1] = c2[q][2] = c2[q][3] = 0.f;
    const __nv_bfloat16 *a2r0 = DA2T + (int64_t)(mt * 16 + gid) * n32, *a2r1 = a2r0 + 8LL * n32;
    const __nv_bfloat16 *a1r0 = DA1T + (int64_t)(mt * 16 + gid) * n32, *a1r1 = a1r0 + 8LL * n32;
    const __nv_bfloat16 *xr = XT + (int64_t)(nq * 8 + gid) * n32;
    for (int k0 = k_begin; k0 < k_end; k0 += 16) {
        const int c = k0 + tig * 2;
        const uint32_t a[4] = {ld_u32(a2r0 + c), ld_u32(a2r1 + c), ld_u32(a2r0 + c + 8),
                               ld_u32(a2r1 + c + 8)};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const __nv_bfloat16 *hr = H1T + (int64_t)((nq * 4 + q) * 8 + gid) * n32;
            const uint32_t b[2] = {ld_u32(hr + c), ld_u32(hr + c + 8)};
            mma_bf16_16816(c2[q], a, b);
        }
        const uint32_t a1[4] = {ld_u32(a1r0 + c), ld_u32(a1r1 + c), ld_u32(a1r0 + c + 8),
                                ld_u32(a1r1 + c + 8)};
        const uint32_t b1[2] = {ld_u32(xr + c), ld_u32(xr + c + 8)};
        mma_bf16_16816(c1, a1, b1);
    }
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const int row = mt * 16 + gid + 8 * (e >> 1);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int col = (nq * 4 + q) * 8 + tig * 2 + (e & 1);
            atomicAdd(grad + kOffW2 + row * kH + col, c2[q][e]);
        }
        const int col1 = nq * 8 + tig * 2 + (e & 1);
        if (col1 < kIn) atomicAdd(grad + kOffW1 + row * kIn + col1, c1[e]);
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

extern "C" int64_t cnb_mlp_grad_mma_scratch_bytes(int n) {
    if (n < 1) return -1;
    const int64_t n32 = ((int64_t)n + 31) / 32 * 32;
    return (16 + 3 * kH) * n32 * (int64_t)sizeof(__nv_bfloat16);
}

extern "C" int cnb_mlp_grad_mma(const float *features, const float *labels, int n,
                                const float *weights, float over_weight, void *scratch,
                                int64_t scratch_bytes, float *grad, float *loss, void *stream) {
    if (n < 1 || !features || !labels || !weights || !scratch || !grad || !loss)
        return CNB_E_INVALID_ARG;
    if ((reinterpret_cast<uintptr_t>(scratch) & 15) != 0 ||
        scratch_bytes < cnb_mlp_grad_mma_scratch_bytes(n))
        return CNB_E_INVALID_ARG;
    if (n > (1 << 28)) return CNB_E_TOO_LARGE;
    cudaStream_t st = as_stream(stream);
    const int n32 = (n + 31) / 32 * 32;
    __nv_bfloat16 *XT = static_cast<__nv_bfloat16 *>(scratch);
    __nv_bfloat16 *H1T = XT + 16LL * n32, *DA2T = H1T + (int64_t)kH * n32,
                  *DA1T = DA2T + (int64_t)kH * n32;
    CNB_CUDA(cudaMemsetAsync(grad, 0, sizeof(float) * kParams, st));
    CNB_CUDA(cudaMemsetAsync(loss, 0, sizeof(float), st));
    CNB_CUDA(cudaFuncSetAttribute(k_mlp_train_mma, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  kTSmem));
    const int tiles = n32 / 32;
    const int blocks = (tiles + kTW - 1) / kTW < 148 * 2 ? (tiles + kTW - 1) / kTW : 148 * 2;
    k_mlp_train_mma<<<blocks, kTW * 32, kTSmem, st>>>(features, labels, n, n32, weights,
                                                       over_weight, XT, H1T, DA2T, DA1T, grad,
                                                       loss);
    CNB_TRY(launch_status());
    constexpr int kChunk = 1024;
    k_mlp_param_mma<<<(n32 + kChunk - 1) / kChunk, kPW * 32, 0, st>>>(XT, H1T, DA2T, DA1T, n32,
                                                                      kChunk, grad);
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
