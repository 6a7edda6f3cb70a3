// grouped.cuh -- parameters and force-list helpers shared by the grouped
// traversals (forces_grouped.cu: bucket opening tests and the periodic law;
// forces_exact.cu: the reference's per-body opening decisions).
#pragma once
#include "common.cuh"

namespace cnb {

constexpr int kGStack = 512;   // node stack entries per warp (deepest seen at 128^3: ~320)
constexpr int kGList = 64;     // interaction list entries per warp

struct GroupedParams {
    const float *px, *py, *pz;
    const float4 *rec;   // [2*M]: (com, mass), (x-extent, 3-D extent, child0 bits, child1 bits)
    const float4 *aabb;  // [2*M]: (min, 0), (max, 0)
    float *force;        // [N,3]
    int32_t *ws;         // [0] bucket count, [1] work counter, [2] max stack depth
    const int4 *buckets; // (first body, count, subtree node, 0)
    const float *theta_per_bucket;  // may be null
    float theta;
    double theta_sq;  // theta^2 in float64, the reference's theta_sq (per-body decisions)
    float G, soft2, box;
    float slab_mass;  // CNB_MAC_PERIODIC: image-ambiguous nodes up to this mass are accepted
    int mac;
    int64_t n;
    int64_t m_nodes;
    int32_t root;
    // many boxes in one tree (boxes.cu): box = codes[first body] >> box_shift
    const uint64_t *codes;      // null: one box
    int box_shift;
    const int32_t *box_roots;   // subtree root per box
    const float4 *box_params;   // (theta, softening, slab mass, 0) per box
    int32_t *bucket_inter;      // per bucket slot: interactions of each of its bodies (may be null)
    const int32_t *bucket_order;  // the order buckets are handed out in (may be null: slot order)
    int test_spill_every;         // exact traversal, tests only: give up on every n-th bucket
    unsigned long long *stats;  // [0] body-node interactions, [1] node tests,
                                // [2] interactions needing the per-pair image (may be null)
    int32_t *status;
    // two-level traversal: the bucket's super-bucket (k_super_lists) has already
    // walked the top of the tree; null = walk from the root
    const int32_t *super_of_body;  // super-bucket slot per body (-1: none)
    const int4 *super_hdr;         // per super-bucket: (same-image, per-pair, near, complete)
    const float4 *far_lists;       // per super-bucket: far_cap entries, same-image ones from the
                                   // front, per-pair ones from the back
    const int32_t *near_lists;     // per super-bucket: near_cap nodes left to each bucket
    int far_cap, near_cap;
    // CNB_MAC_EWALD: g and its Jacobian on the octant grid (cnb_ewald_table)
    const float4 *ewald;
    int ewald_nt;
    // CNB_MAC_EWALD: second central moments of internal nodes (two float4 per
    // node, cnb_upward_table_quad), null = monopoles only
    const float4 *quad;
};

// Nearest-image offset of a coordinate difference d with |d| < 1.5: -1, 0
// or +1 (ties at +-0.5 round to 0), i.e. rint(d) -- one instruction where a
// compare-and-select chain takes four per axis.
__device__ __forceinline__ float image_of(float d) { return rintf(d); }

// The same offset by compare-and-select, on the FP32 / ALU pipes: the per-pair
// form of the force loop, where rint on the XU pipe would compete with rsqrt.
__device__ __forceinline__ float pair_image(float d) {
    return d > 0.5f ? 1.f : (d < -0.5f ? -1.f : 0.f);
}

// The reference's cut d^2 > 1e-7 can only drop a pair whose node lies within
// sqrt(1e-7) of the bucket's box.  The walk sends every accepted entry whose
// distance^2 to the box is at most kCutGuard (twice the cut: a margin far
// above the rounding of the box distance) to the list applied WITH the cut;
// the other entries are at d^2 > 1e-7 from every body of the bucket and skip
// the test.
constexpr float kCutGuard = 2e-7f;

// Exact opening decisions (CNB_MAC_REF_X): a node counts as accepted or
// opened by every body of a box only when float32 rounding cannot change
// that -- distances from the box widened by kBoxSlack (the box's own
// rounding), comparisons with a relative margin of kRelMargin.
constexpr float kBoxSlack = 1e-6f;
constexpr float kRelMargin = 4e-6f;

// Applies cnt list entries (x, y, z, mass) to the lane's BPL bodies.  WRAP:
// the entries' image may differ between the bucket's bodies, so every pair
// takes its own minimum image.  CUT: apply the reference's d^2 > 1e-7 cut.
template <int BPL, bool WRAP, bool CUT>
__device__ __forceinline__ void apply_list(const float4 *list, int cnt, const float (&x)[BPL],
                                           const float (&y)[BPL], const float (&z)[BPL],
                                           float soft2, float (&ax)[BPL], float (&ay)[BPL],
                                           float (&az)[BPL]) {
    // the softening enters the distance chain (d^2 + eps^2 in three FMAs);
    // the reference's cut d^2 > 1e-7 becomes d^2 + eps^2 > eps^2 + 1e-7
    const float cut = soft2 + 1e-7f;
#pragma unroll 4
    for (int j = 0; j < cnt; ++j) {
        const float4 e = list[j];
#pragma unroll
        for (int b = 0; b < BPL; ++b) {
            float dx = e.x - x[b], dy = e.y - y[b], dz = e.z - z[b];
            if (WRAP) {
                dx -= pair_image(dx);
                dy -= pair_image(dy);
                dz -= pair_image(dz);
            }
            const float q = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, soft2)));
            const float r = rsqrtf(q);
            const float f = (!CUT || q > cut) ? e.w * r * r * r : 0.f;
            ax[b] = fmaf(f, dx, ax[b]);
            ay[b] = fmaf(f, dy, ay[b]);
            az[b] = fmaf(f, dz, az[b]);
        }
    }
}

// Two bodies per lane: the interaction list holds every entry twice over
// (x, x, y, y | z, z, m, m), so a lane's two bodies form packed float2
// operands and each FP32 instruction (FADD2 / FMUL2 / FFMA2, sm_100) serves
// both.  The arithmetic, and its order, is the scalar loop's, so the forces
// are bit-identical to it; only the minimum image is formed differently
// (d - rint(d) through the 1.5 * 2^23 rounding constant, equal to pair_image
// on |d| < 1.5).
template <bool WRAP, bool CUT>
__device__ __forceinline__ void apply_list_pair(const float4 *list, int cnt, const float (&x)[2],
                                                const float (&y)[2], const float (&z)[2],
                                                float soft2, float (&ax)[2], float (&ay)[2],
                                                float (&az)[2]) {
    const float2 nx = make_float2(-x[0], -x[1]), ny = make_float2(-y[0], -y[1]),
                 nz = make_float2(-z[0], -z[1]);
    const float2 s2 = make_float2(soft2, soft2);
    const float cut = soft2 + 1e-7f;  // the reference's d^2 > 1e-7 on d^2 + eps^2
    const float2 rc = make_float2(12582912.f, 12582912.f), nrc = make_float2(-12582912.f, -12582912.f);
    const float2 m1 = make_float2(-1.f, -1.f);
    float2 fx = make_float2(ax[0], ax[1]), fy = make_float2(ay[0], ay[1]),
           fz = make_float2(az[0], az[1]);
    // eight entries at a time: their loads, distances and inverse cubes are
    // independent, then they are accumulated in list order
    int j = 0;
    for (; j + 8 <= cnt; j += 8) {
        float2 dx[8], dy[8], dz[8], w[8], d2[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const float4 a = list[2 * (j + u)], b = list[2 * (j + u) + 1];
            dx[u] = __fadd2_rn(make_float2(a.x, a.y), nx);
            dy[u] = __fadd2_rn(make_float2(a.z, a.w), ny);
            dz[u] = __fadd2_rn(make_float2(b.x, b.y), nz);
            w[u] = make_float2(b.z, b.w);
            if (WRAP) {
                dx[u] = __ffma2_rn(__fadd2_rn(__fadd2_rn(dx[u], rc), nrc), m1, dx[u]);
                dy[u] = __ffma2_rn(__fadd2_rn(__fadd2_rn(dy[u], rc), nrc), m1, dy[u]);
                dz[u] = __ffma2_rn(__fadd2_rn(__fadd2_rn(dz[u], rc), nrc), m1, dz[u]);
            }
            d2[u] = __ffma2_rn(dx[u], dx[u], __ffma2_rn(dy[u], dy[u], __ffma2_rn(dz[u], dz[u], s2)));
        }
        float2 f[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const float2 q = d2[u];
            float r0 = rsqrtf(q.x), r1 = rsqrtf(q.y);
            if (CUT) {
                r0 = q.x > cut ? r0 : 0.f;
                r1 = q.y > cut ? r1 : 0.f;
            }
            const float2 r = make_float2(r0, r1);
            f[u] = __fmul2_rn(__fmul2_rn(__fmul2_rn(w[u], r), r), r);
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            fx = __ffma2_rn(f[u], dx[u], fx);
            fy = __ffma2_rn(f[u], dy[u], fy);
            fz = __ffma2_rn(f[u], dz[u], fz);
        }
    }
    for (; j < cnt; ++j) {
        const float4 a = list[2 * j], b = list[2 * j + 1];
        float2 dx = __fadd2_rn(make_float2(a.x, a.y), nx);
        float2 dy = __fadd2_rn(make_float2(a.z, a.w), ny);
        float2 dz = __fadd2_rn(make_float2(b.x, b.y), nz);
        if (WRAP) {
            dx = __ffma2_rn(__fadd2_rn(__fadd2_rn(dx, rc), nrc), m1, dx);
            dy = __ffma2_rn(__fadd2_rn(__fadd2_rn(dy, rc), nrc), m1, dy);
            dz = __ffma2_rn(__fadd2_rn(__fadd2_rn(dz, rc), nrc), m1, dz);
        }
        const float2 q = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __ffma2_rn(dz, dz, s2)));
        float r0 = rsqrtf(q.x), r1 = rsqrtf(q.y);
        if (CUT) {
            r0 = q.x > cut ? r0 : 0.f;
            r1 = q.y > cut ? r1 : 0.f;
        }
        const float2 r = make_float2(r0, r1);
        const float2 f = __fmul2_rn(__fmul2_rn(__fmul2_rn(make_float2(b.z, b.w), r), r), r);
        fx = __ffma2_rn(f, dx, fx);
        fy = __ffma2_rn(f, dy, fy);
        fz = __ffma2_rn(f, dz, fz);
    }
    ax[0] = fx.x; ax[1] = fx.y;
    ay[0] = fy.x; ay[1] = fy.y;
    az[0] = fz.x; az[1] = fz.y;
}

// float4 slots per list entry
template <int BPL> __host__ __device__ constexpr int entry_width() { return BPL == 2 ? 2 : 1; }

template <int BPL>
__device__ __forceinline__ void put_entry(float4 *list, int idx, float4 e) {
    if (BPL == 2) {
        list[2 * idx] = make_float4(e.x, e.x, e.y, e.y);
        list[2 * idx + 1] = make_float4(e.z, e.z, e.w, e.w);
    } else {
        list[idx] = e;
    }
}

template <int BPL, bool WRAP, bool CUT>
__device__ __forceinline__ void apply_entries(const float4 *list, int cnt, const float (&x)[BPL],
                                              const float (&y)[BPL], const float (&z)[BPL],
                                              float soft2, float (&ax)[BPL], float (&ay)[BPL],
                                              float (&az)[BPL]) {
    if constexpr (BPL == 2)
        apply_list_pair<WRAP, CUT>(list, cnt, x, y, z, soft2, ax, ay, az);
    else
        apply_list<BPL, WRAP, CUT>(list, cnt, x, y, z, soft2, ax, ay, az);
}

// forces_exact.cu: the grouped traversal with the reference's per-body
// opening decisions (CNB_MAC_REF_X); P.ws[1] must be zero.
int launch_exact(GroupedParams &P, int bodies_per_lane, int block_warps, cudaStream_t st);

}  // namespace cnb
