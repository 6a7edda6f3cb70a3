// morton.cu -- Morton keys (src/kernels/morton.py:13-90).
//
// HBM-bound streaming kernel: 12 B read + 8 B key (+4 B index) written per
// particle.  Four particles per thread through 128-bit loads/stores when the
// arrays are 16-byte aligned.
#include "common.cuh"

namespace cnb {

// morton.py:13-37: the reference's masks (they keep the low 10 bits).
__device__ __forceinline__ uint64_t spread_compat(uint64_t v) {
    v = (v | (v << 16)) & 0x030000FFull;
    v = (v | (v << 8)) & 0x0300F00Full;
    v = (v | (v << 4)) & 0x030C30C3ull;
    v = (v | (v << 2)) & 0x09249249ull;
    return v;
}

// Full 21-bit spread: bit b of v goes to bit 3b.
__device__ __forceinline__ uint64_t spread21(uint64_t v) {
    v &= 0x1fffffull;
    v = (v | (v << 32)) & 0x001f00000000ffffull;
    v = (v | (v << 16)) & 0x001f0000ff0000ffull;
    v = (v | (v << 8)) & 0x100f00f00f00f00full;
    v = (v | (v << 4)) & 0x10c30c30c30c30c3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}

// morton.py:57-59: uint64(x * 2^21) with x promoted to float64 (exact),
// truncated; negative / NaN -> 0.
__device__ __forceinline__ uint64_t scale21(float x) {
    double s = (double)x * 2097152.0;
    if (!(s > 0.0)) return 0ull;
    if (s >= 18446744073709551615.0) return ~0ull;
    return __double2ull_rz(s);
}

template <int MODE>
__device__ __forceinline__ uint64_t morton_key(float x, float y, float z) {
    uint64_t ix = scale21(x), iy = scale21(y), iz = scale21(z);
    if (MODE == CNB_KEY_COMPAT30) {
        return spread_compat(ix) | (spread_compat(iy) << 1) | (spread_compat(iz) << 2);
    } else {
        const uint64_t lim = (1ull << 21) - 1;
        ix = ix > lim ? lim : ix;
        iy = iy > lim ? lim : iy;
        iz = iz > lim ? lim : iz;
        return spread21(ix) | (spread21(iy) << 1) | (spread21(iz) << 2);
    }
}

template <int MODE>
__global__ void __launch_bounds__(256) k_codes_vec4(const float4 *__restrict__ x,
                                                    const float4 *__restrict__ y,
                                                    const float4 *__restrict__ z,
                                                    ulonglong2 *__restrict__ codes,
                                                    uint4 *__restrict__ idx, int64_t n4) {
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n4;
         q += (int64_t)gridDim.x * blockDim.x) {
        float4 a = __ldcs(x + q), b = __ldcs(y + q), c = __ldcs(z + q);
        ulonglong2 k0, k1;
        k0.x = morton_key<MODE>(a.x, b.x, c.x);
        k0.y = morton_key<MODE>(a.y, b.y, c.y);
        k1.x = morton_key<MODE>(a.z, b.z, c.z);
        k1.y = morton_key<MODE>(a.w, b.w, c.w);
        codes[2 * q] = k0;
        codes[2 * q + 1] = k1;
        if (idx) {
            uint32_t i0 = (uint32_t)(4 * q);
            idx[q] = make_uint4(i0, i0 + 1, i0 + 2, i0 + 3);
        }
    }
}

template <int MODE>
__global__ void __launch_bounds__(256) k_codes_scalar(const float *__restrict__ x,
                                                      const float *__restrict__ y,
                                                      const float *__restrict__ z,
                                                      uint64_t *__restrict__ codes,
                                                      uint32_t *__restrict__ idx, int64_t lo,
                                                      int64_t n) {
    for (int64_t i = lo + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        codes[i] = morton_key<MODE>(x[i], y[i], z[i]);
        if (idx) idx[i] = (uint32_t)i;
    }
}

template <int MODE>
static int launch_codes(const float *x, const float *y, const float *z, uint64_t *codes,
                        uint32_t *idx, int64_t n, cudaStream_t st) {
    auto al = [](const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; };
    int64_t done = 0;
    if (n >= 4 && al(x) && al(y) && al(z) && al(codes) && (idx == nullptr || al(idx))) {
        int64_t n4 = n / 4;
        k_codes_vec4<MODE><<<grid_for(n4, 256, 148 * 16), 256, 0, st>>>(
            reinterpret_cast<const float4 *>(x), reinterpret_cast<const float4 *>(y),
            reinterpret_cast<const float4 *>(z), reinterpret_cast<ulonglong2 *>(codes),
            reinterpret_cast<uint4 *>(idx), n4);
        CNB_TRY(launch_status());
        done = n4 * 4;
    }
    if (done < n) {
        k_codes_scalar<MODE><<<grid_for(n - done, 256, 148 * 16), 256, 0, st>>>(x, y, z, codes,
                                                                                 idx, done, n);
        CNB_TRY(launch_status());
    }
    return CNB_OK;
}

}  // namespace cnb

extern "C" int cnb_compute_codes(const float *x, const float *y, const float *z,
                                 uint64_t *codes, uint32_t *indices, int64_t n, int key_mode,
                                 void *stream) {
    if (n < 0 || (n > 0 && (!x || !y || !z || !codes))) return CNB_E_INVALID_ARG;
    if (n > (int64_t)UINT32_MAX) return CNB_E_TOO_LARGE;
    if (n == 0) return CNB_OK;
    cudaStream_t st = cnb::as_stream(stream);
    if (key_mode == CNB_KEY_COMPAT30)
        return cnb::launch_codes<CNB_KEY_COMPAT30>(x, y, z, codes, indices, n, st);
    if (key_mode == CNB_KEY_MORTON63)
        return cnb::launch_codes<CNB_KEY_MORTON63>(x, y, z, codes, indices, n, st);
    return CNB_E_INVALID_ARG;
}
