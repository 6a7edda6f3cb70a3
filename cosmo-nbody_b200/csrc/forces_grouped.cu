// forces_grouped.cu -- warp-cooperative Barnes-Hut traversal over
// Morton-contiguous buckets (the B200 form of
// src/kernels/physics_kernels.py:14-153).
//
// A bucket is a maximal radix-tree subtree with at most 32*BPL bodies
// (cnb_make_buckets), so it is contiguous in the sorted order and spatially
// compact.  One warp takes a bucket (dynamic scheduling: an atomic work
// counter), each lane holds BPL bodies.  The warp walks the tree 32 nodes at
// a time from a per-warp node stack in shared memory: each lane tests one
// node against the bucket's bounding box, accepted nodes (and reached
// leaves) are appended to a per-warp interaction list in shared memory with
// one ballot, opened nodes push their two children.  Whenever the list holds
// 32 entries, every lane applies them to its bodies: float32, rsqrt, and the
// per-pair minimum image only for entries whose image can differ between the
// bucket's bodies (flagged by a negative mass), so the force loop reads
// shared memory only and never diverges.  The reference's cut (no force from a
// node at d^2 <= 1e-7) is tested only on the second list's entries: those
// with a per-pair image and those within sqrt(2e-7) of the bucket's box, the
// only ones the cut can reach.
//
// Opening tests (bucket box B with centre g and half-size h, node CoM image c
// nearest g, dmin = periodic distance from c to B, per axis):
//   CNB_MAC_REF_X:    open unless leaf or sx^2 < theta^2 dmin^2, sx the node's
//                     x-extent set to `box` above box/2 (physics_kernels.py:131-136).
//                     Each node the bucket accepts, every one of its bodies
//                     would accept in the reference traversal (dmin <= |d|).
//   CNB_MAC_PERIODIC: 3-D extent l; also open any node whose members' image is
//                     not the same for every body of the bucket, so an accepted
//                     monopole is applied at one consistent image -- unless the
//                     node's mass is at most slab_mass, when it is applied with
//                     the per-pair minimum image of its CoM.  slab_mass = 0 is
//                     exact; a small positive value bounds the cost of the
//                     sources near the plane antipodal to the bucket.
//   CNB_MAC_EWALD:    the periodic (Ewald) force law (the EWALD variant of the
//                     kernel): 3-D extent, or b_max with quadrupoles; every
//                     accepted node at the image nearest the bucket centre for
//                     the whole bucket, plus the periodic correction of every
//                     accepted node, accumulated per lane while walking and
//                     applied per body once per bucket (ewald.cu has the law).
//                     With quadrupole moments the second list carries the
//                     internal nodes with their second central moments (and
//                     the first list keeps the cut); without, the entries near
//                     the bucket's box (the cut's).
// theta is one value or one per bucket (learned controller).
//
// Two bodies per lane run the force loop on packed float2 (FADD2 / FMUL2 /
// FFMA2); the two-level walk (k_super_lists, cnb_forces_two_level) lets a
// super-bucket walk the top of the tree once for all its buckets.
#include "grouped.cuh"

namespace cnb {


// Periodic correction of one accepted node, d = its CoM image minus the
// bucket centre (|d_i| <= 1/2): g(d) and its Jacobian from the nearest
// point of the octant table, g to first order about that point, signs from
// g's symmetry (g_i odd in d_i, even in the other components).
__device__ __forceinline__ void ewald_lookup(const float4 *__restrict__ T, int nt, float dx,
                                             float dy, float dz, float (&g)[3], float (&J)[6]) {
    const float ax = fabsf(dx), ay = fabsf(dy), az = fabsf(dz);
    const float sc = 2.f * nt;
    const int i = min(__float2int_rn(ax * sc), nt), j = min(__float2int_rn(ay * sc), nt),
              k = min(__float2int_rn(az * sc), nt);
    const int64_t t = ((int64_t)i * (nt + 1) + j) * (nt + 1) + k;
    const float4 t0 = __ldg(T + 6 * t), t1 = __ldg(T + 6 * t + 1), t2 = __ldg(T + 6 * t + 2);
    const float h = 1.f / sc;
    const float ex = ax - i * h, ey = ay - j * h, ez = az - k * h;
    // octant: g(a) = g(a0) + J(a0) (a - a0); J = (xx, xy, xz, yy, yz, zz)
    const float gx = t0.x + t1.x * ex + t1.y * ey + t1.z * ez;
    const float gy = t0.y + t1.y * ex + t1.w * ey + t2.x * ez;
    const float gz = t0.z + t1.z * ex + t2.x * ey + t2.y * ez;
    const float sx = dx < 0.f ? -1.f : 1.f, sy = dy < 0.f ? -1.f : 1.f, sz = dz < 0.f ? -1.f : 1.f;
    g[0] = sx * gx;
    g[1] = sy * gy;
    g[2] = sz * gz;
    J[0] = t1.x;
    J[1] = sx * sy * t1.y;
    J[2] = sx * sz * t1.z;
    J[3] = t1.w;
    J[4] = sy * sz * t2.x;
    J[5] = t2.y;
}

// The periodic part of a node's quadrupole force, (1/2) H(d) : M2, with H
// (the second derivatives of g) at the table point nearest d and M2 the
// node's second central moment (xx, xy, xz, yy | yz, zz).
__device__ __forceinline__ void ewald_quad(const float4 *__restrict__ T, int nt, float dx, float dy,
                                           float dz, float4 ma, float4 mb, float (&out)[3]) {
    const float sc = 2.f * nt;
    const int i = min(__float2int_rn(fabsf(dx) * sc), nt), j = min(__float2int_rn(fabsf(dy) * sc), nt),
              k = min(__float2int_rn(fabsf(dz) * sc), nt);
    const int64_t t = ((int64_t)i * (nt + 1) + j) * (nt + 1) + k;
    const float4 h0 = __ldg(T + 6 * t + 3), h1 = __ldg(T + 6 * t + 4), h2 = __ldg(T + 6 * t + 5);
    const float sx = dx < 0.f ? -1.f : 1.f, sy = dy < 0.f ? -1.f : 1.f, sz = dz < 0.f ? -1.f : 1.f;
    // H_ijk(d) = s_i s_j s_k H_ijk(|d|)
    const float xxx = sx * h0.x, xxy = sy * h0.y, xxz = sz * h0.z, xyy = sx * h0.w;
    const float xyz = sx * sy * sz * h1.x, xzz = sx * h1.y, yyy = sy * h1.z, yyz = sz * h1.w;
    const float yzz = sy * h2.x, zzz = sz * h2.y;
    const float mxx = ma.x, mxy = ma.y, mxz = ma.z, myy = ma.w, myz = mb.x, mzz = mb.y;
    // (1/2) sum_jk H_ijk M_jk, off-diagonal pairs counted twice
    out[0] = 0.5f * (xxx * mxx + xyy * myy + xzz * mzz) + xxy * mxy + xxz * mxz + xyz * myz;
    out[1] = 0.5f * (xxy * mxx + yyy * myy + yzz * mzz) + xyy * mxy + xyz * mxz + yyz * myz;
    out[2] = 0.5f * (xxz * mxx + yyz * myy + zzz * mzz) + xyz * mxy + xzz * mxz + yzz * myz;
}


// float4 slots per entry of the second list: the per-pair-image list, or
// under the periodic law the quadrupole list (position and mass | xx, xy, xz,
// yy | yz, zz, trace, 0 of the node's second central moment)
template <int BPL, bool EWALD> __host__ __device__ constexpr int second_width() {
    return EWALD ? 3 : entry_width<BPL>();
}

// The exact minimum-image test (CNB_MAC_PERIODIC) opens every node whose
// image box can reach a bucket and walks far wider than the other tests:
// its node stack is this many entries per warp.
constexpr int kGStackPeriodic = 4096;

template <int BPL, bool EWALD>
constexpr size_t grouped_smem(int warps, int stack) {
    return (size_t)warps * (stack * sizeof(int32_t) +
                            kGList * (entry_width<BPL>() + second_width<BPL, EWALD>()) *
                                sizeof(float4));
}

// Applies cnt quadrupole entries: per body the softened monopole plus
// (15/2)(d.M d) d / r^7 - 3 M d / r^5 - (3/2) tr(M) d / r^5 for the node's
// second central moment M about its CoM (d = CoM - body, r softened).
template <int BPL>
__device__ __forceinline__ void apply_quad(const float4 *q, int cnt, const float (&x)[BPL],
                                           const float (&y)[BPL], const float (&z)[BPL],
                                           float soft2, float (&ax)[BPL], float (&ay)[BPL],
                                           float (&az)[BPL]) {
    const float cut = soft2 + 1e-7f;
    if constexpr (BPL == 2) {
        // two bodies per lane as packed float2 (FADD2 / FMUL2 / FFMA2)
        const float2 nx = make_float2(-x[0], -x[1]), ny = make_float2(-y[0], -y[1]),
                     nz = make_float2(-z[0], -z[1]);
        const float2 s2 = make_float2(soft2, soft2);
        float2 fx = make_float2(ax[0], ax[1]), fy = make_float2(ay[0], ay[1]),
               fz = make_float2(az[0], az[1]);
        const auto dup = [](float a) { return make_float2(a, a); };
#pragma unroll 2
        for (int j = 0; j < cnt; ++j) {
            const float4 e = q[3 * j], u = q[3 * j + 1], v = q[3 * j + 2];
            const float2 dx = __fadd2_rn(dup(e.x), nx), dy = __fadd2_rn(dup(e.y), ny),
                         dz = __fadd2_rn(dup(e.z), nz);
            const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __ffma2_rn(dz, dz, s2)));
            const float2 ri = make_float2(rsqrtf(r2.x), rsqrtf(r2.y));
            const float2 ri2 = __fmul2_rn(ri, ri), ri3 = __fmul2_rn(ri2, ri);
            const float2 ri5 = __fmul2_rn(ri3, ri2), ri7 = __fmul2_rn(ri5, ri2);
            const float2 qx = __ffma2_rn(dup(u.x), dx, __ffma2_rn(dup(u.y), dy, __fmul2_rn(dup(u.z), dz)));
            const float2 qy = __ffma2_rn(dup(u.y), dx, __ffma2_rn(dup(u.w), dy, __fmul2_rn(dup(v.x), dz)));
            const float2 qz = __ffma2_rn(dup(u.z), dx, __ffma2_rn(dup(v.x), dy, __fmul2_rn(dup(v.y), dz)));
            const float2 sq = __ffma2_rn(dx, qx, __ffma2_rn(dy, qy, __fmul2_rn(dz, qz)));
            float2 A = __ffma2_rn(dup(e.w), ri3,
                                  __ffma2_rn(__fmul2_rn(dup(7.5f), sq), ri7, __fmul2_rn(dup(-1.5f * v.z), ri5)));
            float2 B = __fmul2_rn(dup(-3.f), ri5);
            if (!(r2.x > cut)) A.x = B.x = 0.f;
            if (!(r2.y > cut)) A.y = B.y = 0.f;
            fx = __ffma2_rn(A, dx, __ffma2_rn(B, qx, fx));
            fy = __ffma2_rn(A, dy, __ffma2_rn(B, qy, fy));
            fz = __ffma2_rn(A, dz, __ffma2_rn(B, qz, fz));
        }
        ax[0] = fx.x; ax[1] = fx.y;
        ay[0] = fy.x; ay[1] = fy.y;
        az[0] = fz.x; az[1] = fz.y;
        return;
    }
#pragma unroll 2
    for (int j = 0; j < cnt; ++j) {
        const float4 e = q[3 * j], u = q[3 * j + 1], v = q[3 * j + 2];
#pragma unroll
        for (int b = 0; b < BPL; ++b) {
            const float dx = e.x - x[b], dy = e.y - y[b], dz = e.z - z[b];
            const float r2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, soft2)));
            const float ri = rsqrtf(r2);
            const float ri2 = ri * ri, ri3 = ri2 * ri, ri5 = ri3 * ri2, ri7 = ri5 * ri2;
            const float qx = fmaf(u.x, dx, fmaf(u.y, dy, u.z * dz));
            const float qy = fmaf(u.y, dx, fmaf(u.w, dy, v.x * dz));
            const float qz = fmaf(u.z, dx, fmaf(v.x, dy, v.y * dz));
            const float sq = fmaf(dx, qx, fmaf(dy, qy, dz * qz));
            float A = fmaf(e.w, ri3, fmaf(7.5f * sq, ri7, -1.5f * v.z * ri5));
            float B = -3.f * ri5;
            if (!(r2 > cut)) A = B = 0.f;
            ax[b] = fmaf(A, dx, fmaf(B, qx, ax[b]));
            ay[b] = fmaf(A, dy, fmaf(B, qy, ay[b]));
            az[b] = fmaf(A, dz, fmaf(B, qz, az[b]));
        }
    }
}

// LAW: 0 the minimum-image laws (CNB_MAC_REF_X, CNB_MAC_PERIODIC), 1 the
// periodic (Ewald) law with monopoles, 2 the periodic law with quadrupoles.
template <int BPL, int WARPS, int LAW, int STACK>
__global__ void __launch_bounds__(WARPS * 32) k_forces_grouped(GroupedParams P) {
    constexpr bool EWALD = LAW != 0;
    constexpr bool QUAD = LAW == 2;
    extern __shared__ __align__(16) unsigned char g_smem[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const uint32_t lt = (1u << lane) - 1u;
    // two interaction lists per warp: entries with one image for the whole
    // bucket, and entries needing the per-pair image (under the periodic law:
    // internal nodes with their quadrupole moments)
    constexpr int EW = entry_width<BPL>();
    constexpr int SW = second_width<BPL, EWALD>();
    float4 *list = reinterpret_cast<float4 *>(g_smem) + wib * kGList * (EW + SW);
    float4 *wlist = list + kGList * EW;
    int32_t *stack =
        reinterpret_cast<int32_t *>(g_smem + WARPS * kGList * (EW + SW) * sizeof(float4)) +
        wib * STACK;
    unsigned long long n_tests = 0;
    int max_top = 0;
    bool overflow = false;
    const int n_buckets = P.ws[0];
    const float half_box = 0.5f * P.box;

    for (;;) {
        int g = 0;
        if (lane == 0) g = atomicAdd(P.ws + 1, 1);
        g = __shfl_sync(0xffffffffu, g, 0);
        if (g >= n_buckets) break;
        if (P.bucket_order) g = P.bucket_order[g];
        const int4 bk = P.buckets[g];
        const int count = bk.y;
        float x[BPL], y[BPL], z[BPL];
        bool valid[BPL];
        float lx = INFINITY, ly = INFINITY, lz = INFINITY;
        float hx = -INFINITY, hy = -INFINITY, hz = -INFINITY;
#pragma unroll
        for (int b = 0; b < BPL; ++b) {
            const int k = lane + 32 * b;
            valid[b] = k < count;
            const int64_t i = (int64_t)bk.x + (valid[b] ? k : 0);
            x[b] = P.px[i];
            y[b] = P.py[i];
            z[b] = P.pz[i];
            if (valid[b]) {
                if (!(isfinite(x[b]) && isfinite(y[b]) && isfinite(z[b])))
                    set_flag(P.status, CNB_FLAG_NONFINITE);
                lx = fminf(lx, x[b]); ly = fminf(ly, y[b]); lz = fminf(lz, z[b]);
                hx = fmaxf(hx, x[b]); hy = fmaxf(hy, y[b]); hz = fmaxf(hz, z[b]);
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            lx = fminf(lx, __shfl_xor_sync(0xffffffffu, lx, o));
            ly = fminf(ly, __shfl_xor_sync(0xffffffffu, ly, o));
            lz = fminf(lz, __shfl_xor_sync(0xffffffffu, lz, o));
            hx = fmaxf(hx, __shfl_xor_sync(0xffffffffu, hx, o));
            hy = fmaxf(hy, __shfl_xor_sync(0xffffffffu, hy, o));
            hz = fmaxf(hz, __shfl_xor_sync(0xffffffffu, hz, o));
        }
        const float gcx = 0.5f * (lx + hx), gcy = 0.5f * (ly + hy), gcz = 0.5f * (lz + hz);
        const float ghx = 0.5f * (hx - lx), ghy = 0.5f * (hy - ly), ghz = 0.5f * (hz - lz);
        // an entry whose image offset from the centre stays below this needs no per-pair wrap
        const float wlx = 0.5f - ghx - 1e-6f, wly = 0.5f - ghy - 1e-6f, wlz = 0.5f - ghz - 1e-6f;
        float th = P.theta, soft2 = P.soft2, slab_mass = P.slab_mass;
        int32_t root = P.root;
        if (P.box_roots) {
            const uint64_t b = P.codes[bk.x] >> P.box_shift;
            const float4 bp = P.box_params[b];
            root = P.box_roots[b];
            th = bp.x;
            soft2 = bp.y * bp.y;
            slab_mass = bp.z;
        }
        if (P.theta_per_bucket) th = P.theta_per_bucket[g];
        const float th2 = th * th;

        float ax[BPL], ay[BPL], az[BPL];
#pragma unroll
        for (int b = 0; b < BPL; ++b) ax[b] = ay[b] = az[b] = 0.f;
        // EWALD: this lane's share of sum m (c - centre), sum m, sum m g, sum m J
        float ec[4] = {0.f, 0.f, 0.f, 0.f}, eg[3] = {0.f, 0.f, 0.f};
        float ej[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        int top = 1, cnt = 0, wcnt = 0;
        unsigned long long n_entries = 0, n_wrap = 0;
        bool seeded = false;
        if (P.super_of_body) {
            const int sup = P.super_of_body[bk.x];
            const int4 h = sup >= 0 ? P.super_hdr[sup] : make_int4(0, 0, 0, 0);
            if (h.w) {
                // the far field the super-bucket accepted holds for this bucket too
                const float4 *far = P.far_lists + (int64_t)sup * P.far_cap;
                for (int j0 = 0; j0 < h.x; j0 += 32) {
                    const int c = min(32, h.x - j0);
                    if (lane < c) put_entry<BPL>(list, lane, far[j0 + lane]);
                    __syncwarp();
                    apply_entries<BPL, false, false>(list, c, x, y, z, soft2, ax, ay, az);
                    __syncwarp();
                }
                for (int j0 = 0; j0 < h.y; j0 += 32) {
                    const int c = min(32, h.y - j0);
                    if (lane < c) put_entry<BPL>(list, lane, far[P.far_cap - h.y + j0 + lane]);
                    __syncwarp();
                    apply_entries<BPL, true, true>(list, c, x, y, z, soft2, ax, ay, az);
                    __syncwarp();
                }
                n_entries += h.x + h.y;
                n_wrap += h.y;
                // the near nodes it left are this bucket's starting stack
                const int32_t *near = P.near_lists + (int64_t)sup * P.near_cap;
                for (int j = lane; j < h.z; j += 32) stack[j] = near[j];
                top = h.z;
                seeded = true;
            }
        }
        if (!seeded && lane == 0) stack[0] = root;
        __syncwarp();
        // a valid tree pushes every node at most once per bucket: more rounds
        // than nodes means a cyclic topology
        int64_t rounds = 0;
        while (top > 0) {
            if (++rounds > P.m_nodes) {
                if (lane == 0) set_flag(P.status, CNB_FLAG_BAD_TOPOLOGY);
                break;
            }
            const int k = top < 32 ? top : 32;
            top -= k;
            int32_t node = -1;
            if (lane < k) node = stack[top + lane];
            __syncwarp();
            if (node >= P.m_nodes) {
                set_flag(P.status, CNB_FLAG_BAD_TOPOLOGY);
                node = -1;
            }
            bool accept = false, open = false, consistent = true, near_box = false;
            float4 E = make_float4(0.f, 0.f, 0.f, 0.f);
            int32_t c0 = -1, c1 = -1;
            if (node >= 0) {
                // both halves of the record (one 32-byte sector) in flight together
                const float4 A = __ldg(P.rec + 2 * node);
                const float4 S = __ldg(P.rec + 2 * node + 1);
                if (A.w > 0.f) {
                    c0 = __float_as_int(S.z);
                    c1 = __float_as_int(S.w);
                    float dx = A.x - gcx, dy = A.y - gcy, dz = A.z - gcz;
                    const float sx_ = image_of(dx), sy_ = image_of(dy), sz_ = image_of(dz);
                    dx -= sx_;
                    dy -= sy_;
                    dz -= sz_;
                    const float tx = fmaxf(fabsf(dx) - ghx, 0.f);
                    const float ty = fmaxf(fabsf(dy) - ghy, 0.f);
                    const float tz = fmaxf(fabsf(dz) - ghz, 0.f);
                    const float d2min = tx * tx + ty * ty + tz * tz;
                    near_box = d2min <= kCutGuard;
                    if (c0 == -1) {
                        accept = true;
                    } else {
                        if (EWALD) {
                            // periodic law: every image is valid; the node's size is its
                            // 3-D extent, or b_max when quadrupoles are applied
                            accept = S.y * S.y < th2 * d2min;
                        } else if (P.mac == CNB_MAC_REF_X_BUCKET) {
                            const float s = S.x > half_box ? P.box : S.x;
                            accept = s * s < th2 * d2min;
                        } else if (S.y * S.y < th2 * d2min) {
                            // node box at the image chosen for its CoM
                            const float4 lo = __ldg(P.aabb + 2 * node);
                            const float4 hi = __ldg(P.aabb + 2 * node + 1);
                            const float ex = fmaxf(hi.x - sx_, hx) - fminf(lo.x - sx_, lx);
                            const float ey = fmaxf(hi.y - sy_, hy) - fminf(lo.y - sy_, ly);
                            const float ez = fmaxf(hi.z - sz_, hz) - fminf(lo.z - sz_, lz);
                            consistent = ex < half_box && ey < half_box && ez < half_box;
                            // a light image-ambiguous node is applied with the
                            // per-pair minimum image of its CoM (bounded error)
                            accept = consistent || A.w <= slab_mass;
                        }
                        open = !accept;
                    }
                    if (accept) {
                        // under the periodic law one image serves the whole bucket
                        const bool same_image = EWALD || (consistent &&
                            fabsf(dx) < wlx && fabsf(dy) < wly && fabsf(dz) < wlz);
                        E = make_float4(A.x - sx_, A.y - sy_, A.z - sz_, same_image ? A.w : -A.w);
                        if (EWALD) {
                            float g[3], J[6];
                            ewald_lookup(P.ewald, P.ewald_nt, dx, dy, dz, g, J);
                            ec[0] = fmaf(A.w, dx, ec[0]);
                            ec[1] = fmaf(A.w, dy, ec[1]);
                            ec[2] = fmaf(A.w, dz, ec[2]);
                            ec[3] += A.w;
#pragma unroll
                            for (int q = 0; q < 3; ++q) eg[q] = fmaf(A.w, g[q], eg[q]);
#pragma unroll
                            for (int q = 0; q < 6; ++q) ej[q] = fmaf(A.w, J[q], ej[q]);
                        }
                    }
                }
            }
            n_tests += (node >= 0);
            const uint32_t am = __ballot_sync(0xffffffffu, accept);
            const uint32_t om = __ballot_sync(0xffffffffu, open);
            // second list: per-pair image, or (periodic law) an internal node's quadrupole;
            // also every entry near enough to the box for the cut to apply, except with
            // quadrupoles (the first list then keeps the cut)
            const bool to_w = EWALD ? (accept && (QUAD ? c0 != -1 : near_box))
                                    : (accept && (E.w < 0.f || near_box));
            const uint32_t wm = __ballot_sync(0xffffffffu, to_w);
            const uint32_t nm = am & ~wm;
            if (accept) {
                if (to_w) {
                    const int w = wcnt + __popc(wm & lt);
                    if (EWALD && !QUAD) {
                        put_entry<BPL>(wlist, w, E);  // near the box: a monopole with the cut
                    } else if (EWALD) {
                        const float4 qa = __ldg(P.quad + 2 * node), qb = __ldg(P.quad + 2 * node + 1);
                        wlist[3 * w] = E;
                        wlist[3 * w + 1] = qa;
                        wlist[3 * w + 2] = make_float4(qb.x, qb.y, qa.x + qa.w + qb.y, 0.f);
                        // and the periodic part of its quadrupole, a bucket constant
                        float pq[3];
                        ewald_quad(P.ewald, P.ewald_nt, E.x - gcx, E.y - gcy, E.z - gcz, qa, qb, pq);
                        eg[0] += pq[0];
                        eg[1] += pq[1];
                        eg[2] += pq[2];
                    } else {
                        put_entry<BPL>(wlist, w, make_float4(E.x, E.y, E.z, fabsf(E.w)));
                    }
                } else {
                    put_entry<BPL>(list, cnt + __popc(nm & lt), E);
                }
            }
            cnt += __popc(nm);
            wcnt += __popc(wm);
            const int nopen = __popc(om);
            if (top + 2 * nopen > STACK) {
                overflow = true;  // children dropped (flagged)
            } else {
                if (open) {
                    const int pos = top + 2 * __popc(om & lt);
                    stack[pos] = c1;
                    stack[pos + 1] = c0;
                }
                top += 2 * nopen;
                max_top = max(max_top, top);
            }
            __syncwarp();
            if (cnt >= 32) {
                if (QUAD)
                    apply_entries<BPL, false, true>(list, 32, x, y, z, soft2, ax, ay, az);
                else
                    apply_entries<BPL, false, false>(list, 32, x, y, z, soft2, ax, ay, az);
                n_entries += 32;
                __syncwarp();
#pragma unroll
                for (int w = 0; w < EW; ++w)
                    if (lane < cnt - 32) list[EW * lane + w] = list[EW * (32 + lane) + w];
                cnt -= 32;
                __syncwarp();
            }
            if (wcnt >= 32) {
                if (QUAD)
                    apply_quad<BPL>(wlist, 32, x, y, z, soft2, ax, ay, az);
                else if (EWALD)
                    apply_entries<BPL, false, true>(wlist, 32, x, y, z, soft2, ax, ay, az);
                else
                    apply_entries<BPL, true, true>(wlist, 32, x, y, z, soft2, ax, ay, az);
                n_entries += 32;
                n_wrap += 32;
                __syncwarp();
                // float4 slots per entry: quadrupole entries, or the monopole layout
                const int ww = (QUAD) ? SW : EW;
#pragma unroll
                for (int w = 0; w < SW; ++w)
                    if (w < ww && lane < wcnt - 32) wlist[ww * lane + w] = wlist[ww * (32 + lane) + w];
                wcnt -= 32;
                __syncwarp();
            }
        }
        if (QUAD)
            apply_entries<BPL, false, true>(list, cnt, x, y, z, soft2, ax, ay, az);
        else
            apply_entries<BPL, false, false>(list, cnt, x, y, z, soft2, ax, ay, az);
        if (QUAD)
            apply_quad<BPL>(wlist, wcnt, x, y, z, soft2, ax, ay, az);
        else if (EWALD)
            apply_entries<BPL, false, true>(wlist, wcnt, x, y, z, soft2, ax, ay, az);
        else
            apply_entries<BPL, true, true>(wlist, wcnt, x, y, z, soft2, ax, ay, az);
        n_entries += cnt + wcnt;
        n_wrap += wcnt;
        __syncwarp();
        if (EWALD) {
            // bucket totals, then per body the periodic correction of every
            // accepted node: -(4 pi/3) sum m (c - x) + sum m g(c - centre)
            // + sum m J(c - centre) (centre - x)
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
                for (int q = 0; q < 4; ++q) ec[q] += __shfl_xor_sync(0xffffffffu, ec[q], o);
#pragma unroll
                for (int q = 0; q < 3; ++q) eg[q] += __shfl_xor_sync(0xffffffffu, eg[q], o);
#pragma unroll
                for (int q = 0; q < 6; ++q) ej[q] += __shfl_xor_sync(0xffffffffu, ej[q], o);
            }
            const float lin = 4.18879020478639f;  // 4 pi / 3
#pragma unroll
            for (int b = 0; b < BPL; ++b) {
                const float ux = gcx - x[b], uy = gcy - y[b], uz = gcz - z[b];
                // sum m (c - x) = sum m (c - centre) + M (centre - x)
                const float cx = fmaf(ec[3], ux, ec[0]), cy = fmaf(ec[3], uy, ec[1]),
                            cz = fmaf(ec[3], uz, ec[2]);
                ax[b] += eg[0] + ej[0] * ux + ej[1] * uy + ej[2] * uz - lin * cx;
                ay[b] += eg[1] + ej[1] * ux + ej[3] * uy + ej[4] * uz - lin * cy;
                az[b] += eg[2] + ej[2] * ux + ej[4] * uy + ej[5] * uz - lin * cz;
            }
        }
#pragma unroll
        for (int b = 0; b < BPL; ++b) {
            if (valid[b]) {
                const int64_t i = (int64_t)bk.x + lane + 32 * b;
                const float fx = P.G * ax[b], fy = P.G * ay[b], fz = P.G * az[b];
                P.force[3 * i] = fx;
                P.force[3 * i + 1] = fy;
                P.force[3 * i + 2] = fz;
                if (!isfinite(fx) || !isfinite(fy) || !isfinite(fz))
                    set_flag(P.status, CNB_FLAG_NONFINITE);
            }
        }
        if (P.bucket_inter && lane == 0) P.bucket_inter[g] = (int32_t)n_entries;
        if (P.stats && lane == 0) {
            atomicAdd(P.stats, n_entries * (unsigned long long)count);
            atomicAdd(P.stats + 2, n_wrap * (unsigned long long)count);
        }
    }
    if (overflow && lane == 0) set_flag(P.status, CNB_FLAG_LIST_OVERFLOW);
    if (P.stats) {
        for (int o = 16; o > 0; o >>= 1) n_tests += __shfl_xor_sync(0xffffffffu, n_tests, o);
        if (lane == 0) atomicAdd(P.stats + 1, n_tests);
    }
    if (lane == 0) atomicMax(P.ws + 2, max_top);
}

// ---------------------------------------------------------------- two-level
// One warp per super-bucket S (a maximal subtree of at most super_bodies
// bodies) walks the top of the tree once, for every bucket inside S, with the
// reference opening test.  With dmin / dmax the smallest / largest distance
// any point of S's box can have to the node's CoM (per axis, periodic):
//   s^2 <  theta^2 dmin^2  every bucket of S accepts the node  -> far list
//   s^2 >= theta^2 dmax^2  every bucket of S opens it           -> push children
//   otherwise              the bucket decides                   -> near list
// (leaves always go to the far list, as a bucket accepts every leaf it
// reaches).  A bucket b inside S has dmin(S) <= dmin(b) <= dmax(S), so the
// nodes a bucket accepts from S's far list plus its own walk from S's near
// nodes are exactly the nodes it accepts walking from the root.  A far entry
// keeps one image for all of S when S lies within half a box of it on every
// axis (then it is the minimum image for every body of S), otherwise it is
// stored for the per-pair minimum image.  A super-bucket whose lists or stack
// do not fit is marked incomplete; its buckets then walk from the root.
struct SuperParams {
    const float4 *rec, *aabb;
    const int32_t *sws;     // [0] super-bucket count, [1] work counter, [2] incomplete count
    const int4 *supers;     // (first body, count, subtree node, 0)
    int4 *hdr;              // (same-image, per-pair, near, complete) per listed super-bucket
    int32_t *super_of_body; // listed super-bucket of each body, -1 if none
    float4 *far;            // far_cap per super-bucket: same-image from the front, per-pair from the back
    int32_t *near;          // near_cap per super-bucket
    int far_cap, near_cap, max_listed;
    float th2, box, half_box;
    int64_t m_nodes;
    int32_t root;
    unsigned long long *stats;
    int32_t *status;
};

constexpr int kSWarps = 8;

__global__ void __launch_bounds__(kSWarps * 32) k_super_lists(SuperParams P) {
    __shared__ int32_t stacks[kSWarps][kGStack];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const uint32_t lt = (1u << lane) - 1u;
    int32_t *stack = stacks[wib];
    const int64_t n_bodies = (P.m_nodes + 1) / 2;
    int n_sup = P.sws[0];
    if (n_sup < 0 || n_sup > n_bodies) {  // not a super-bucket table of this tree
        if (blockIdx.x == 0 && threadIdx.x == 0) set_flag(P.status, CNB_FLAG_BAD_TOPOLOGY);
        n_sup = 0;
    }
    unsigned long long n_tests = 0;
    for (;;) {
        int s = 0;
        if (lane == 0) s = atomicAdd(const_cast<int32_t *>(P.sws) + 1, 1);
        s = __shfl_sync(0xffffffffu, s, 0);
        if (s >= n_sup) break;
        const int4 sb = P.supers[s];
        if (sb.x < 0 || sb.y < 1 || (int64_t)sb.x + sb.y > n_bodies || sb.z < 0 ||
            sb.z >= P.m_nodes) {
            if (lane == 0) set_flag(P.status, CNB_FLAG_BAD_TOPOLOGY);
            continue;
        }
        const bool listed = s < P.max_listed;
        for (int k = lane; k < sb.y; k += 32) P.super_of_body[sb.x + k] = listed ? s : -1;
        if (!listed) continue;
        const float4 blo = __ldg(P.aabb + 2 * sb.z), bhi = __ldg(P.aabb + 2 * sb.z + 1);
        const float gx = 0.5f * (blo.x + bhi.x), gy = 0.5f * (blo.y + bhi.y), gz = 0.5f * (blo.z + bhi.z);
        // half-sizes widened by kBoxSlack and tests with the margin kRelMargin:
        // a far or opened node is one that every body of S accepts or opens
        // under the reference's float64 test, whatever float32 rounding does
        const float hx = 0.5f * (bhi.x - blo.x) + kBoxSlack, hy = 0.5f * (bhi.y - blo.y) + kBoxSlack,
                    hz = 0.5f * (bhi.z - blo.z) + kBoxSlack;
        const float wlx = 0.5f - hx - 1e-6f, wly = 0.5f - hy - 1e-6f, wlz = 0.5f - hz - 1e-6f;
        float4 *far = P.far + (int64_t)s * P.far_cap;
        int32_t *near = P.near + (int64_t)s * P.near_cap;
        int top = 1, n_same = 0, n_wrap = 0, n_near = 0;
        bool ok = true;
        if (lane == 0) stack[0] = P.root;
        __syncwarp();
        int64_t rounds = 0;
        while (top > 0) {
            if (++rounds > P.m_nodes) {
                if (lane == 0) set_flag(P.status, CNB_FLAG_BAD_TOPOLOGY);
                ok = false;
                break;
            }
            const int k = top < 32 ? top : 32;
            top -= k;
            int32_t node = -1;
            if (lane < k) node = stack[top + lane];
            __syncwarp();
            if (node >= P.m_nodes) {
                set_flag(P.status, CNB_FLAG_BAD_TOPOLOGY);
                node = -1;
            }
            // 1: far, one image   2: far, per-pair image   3: open   4: near
            int cls = 0;
            float4 E = make_float4(0.f, 0.f, 0.f, 0.f);
            int32_t c0 = -1, c1 = -1;
            if (node >= 0) {
                const float4 A = __ldg(P.rec + 2 * node);
                const float4 S = __ldg(P.rec + 2 * node + 1);
                if (A.w > 0.f) {
                    c0 = __float_as_int(S.z);
                    c1 = __float_as_int(S.w);
                    float dx = A.x - gx, dy = A.y - gy, dz = A.z - gz;
                    const float sx_ = image_of(dx), sy_ = image_of(dy), sz_ = image_of(dz);
                    dx -= sx_;
                    dy -= sy_;
                    dz -= sz_;
                    const float adx = fabsf(dx), ady = fabsf(dy), adz = fabsf(dz);
                    const float tx = fmaxf(adx - hx, 0.f), ty = fmaxf(ady - hy, 0.f),
                                tz = fmaxf(adz - hz, 0.f);
                    const float d2min = tx * tx + ty * ty + tz * tz;
                    // the per-pair part also takes every entry near enough to
                    // the box for the reference's cut to apply (it is applied with it)
                    const int far_cls =
                        (adx < wlx && ady < wly && adz < wlz && d2min > kCutGuard) ? 1 : 2;
                    if (c0 == -1) {
                        cls = far_cls;
                    } else {
                        const float s = S.x > P.half_box ? P.box : S.x;
                        if (s * s < P.th2 * d2min * (1.f - kRelMargin)) {
                            cls = far_cls;
                        } else {
                            const float ux = fminf(adx + hx, P.half_box),
                                        uy = fminf(ady + hy, P.half_box),
                                        uz = fminf(adz + hz, P.half_box);
                            cls = (s * s > P.th2 * (ux * ux + uy * uy + uz * uz) * (1.f + kRelMargin))
                                      ? 3 : 4;
                        }
                    }
                    // one image for all of S: the CoM at that image; per pair: the raw
                    // CoM, whose per-pair minimum image is then the reference's own
                    E = cls == 1 ? make_float4(A.x - sx_, A.y - sy_, A.z - sz_, A.w) : A;
                }
            }
            n_tests += (node >= 0);
            const uint32_t m1 = __ballot_sync(0xffffffffu, cls == 1);
            const uint32_t m2 = __ballot_sync(0xffffffffu, cls == 2);
            const uint32_t m3 = __ballot_sync(0xffffffffu, cls == 3);
            const uint32_t m4 = __ballot_sync(0xffffffffu, cls == 4);
            const int c_same = __popc(m1), c_wrap = __popc(m2), c_open = __popc(m3),
                      c_near = __popc(m4);
            if (n_same + c_same + n_wrap + c_wrap > P.far_cap || n_near + c_near > P.near_cap ||
                top + 2 * c_open > kGStack) {
                ok = false;
                break;
            }
            if (cls == 1) far[n_same + __popc(m1 & lt)] = E;
            if (cls == 2) far[P.far_cap - 1 - (n_wrap + __popc(m2 & lt))] = E;
            if (cls == 4) near[n_near + __popc(m4 & lt)] = node;
            if (cls == 3) {
                const int pos = top + 2 * __popc(m3 & lt);
                stack[pos] = c1;
                stack[pos + 1] = c0;
            }
            n_same += c_same;
            n_wrap += c_wrap;
            n_near += c_near;
            top += 2 * c_open;
            __syncwarp();
        }
        __syncwarp();
        if (lane == 0) {
            P.hdr[s] = make_int4(n_same, n_wrap, n_near, ok ? 1 : 0);
            if (!ok) atomicAdd(const_cast<int32_t *>(P.sws) + 2, 1);
        }
    }
    if (P.stats) {
        for (int o = 16; o > 0; o >>= 1) n_tests += __shfl_xor_sync(0xffffffffu, n_tests, o);
        if (lane == 0) atomicAdd(P.stats + 1, n_tests);
    }
}

// Traversal node table from the reference-layout tree: 32-byte records
// (com, mass | x-extent, 3-D extent, children) and the boxes (min | max).
__global__ void __launch_bounds__(256) k_pack_nodes(const float *__restrict__ n_mass,
                                                    const float *__restrict__ n_com,
                                                    const float *__restrict__ n_min,
                                                    const float *__restrict__ n_max,
                                                    const int2 *__restrict__ children,
                                                    float4 *__restrict__ rec,
                                                    float4 *__restrict__ aabb, int64_t m) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int2 ch = children[i];
        const float lx = n_min[3 * i], ly = n_min[3 * i + 1], lz = n_min[3 * i + 2];
        const float hx = n_max[3 * i], hy = n_max[3 * i + 1], hz = n_max[3 * i + 2];
        const float sx = hx - lx;  // physics_kernels.py:131 (before the clamp)
        const float l3 = fmaxf(sx, fmaxf(hy - ly, hz - lz));
        rec[2 * i] = make_float4(n_com[3 * i], n_com[3 * i + 1], n_com[3 * i + 2], n_mass[i]);
        rec[2 * i + 1] = make_float4(sx, l3, __int_as_float(ch.x), __int_as_float(ch.y));
        aabb[2 * i] = make_float4(lx, ly, lz, 0.f);
        aabb[2 * i + 1] = make_float4(hx, hy, hz, 0.f);
    }
}

// Heaviest buckets first: a counting sort of the bucket slots by theta in
// 32 bins over [0.2, 1.0] (smallest theta = most interactions first), so the
// persistent traversal does not end on a few expensive buckets.  One block;
// the order inside a bin is whatever the atomics give (each bucket's result
// does not depend on when it runs).
constexpr int kOrderBins = 32;
__global__ void __launch_bounds__(1024) k_order_buckets(const float *__restrict__ theta,
                                                        const int32_t *__restrict__ ws,
                                                        int32_t *__restrict__ order) {
    __shared__ int32_t cnt[kOrderBins], start[kOrderBins];
    const int nb = ws[0];
    if (threadIdx.x < kOrderBins) cnt[threadIdx.x] = 0;
    __syncthreads();
    auto bin_of = [](float t) {
        const int b = (int)((t - 0.2f) * (kOrderBins / 0.8f));
        return b < 0 ? 0 : (b >= kOrderBins ? kOrderBins - 1 : b);
    };
    for (int g = threadIdx.x; g < nb; g += blockDim.x) atomicAdd(&cnt[bin_of(theta[g])], 1);
    __syncthreads();
    if (threadIdx.x == 0) {
        int run = 0;
        for (int b = 0; b < kOrderBins; ++b) {
            start[b] = run;
            run += cnt[b];
        }
    }
    __syncthreads();
    for (int g = threadIdx.x; g < nb; g += blockDim.x) order[atomicAdd(&start[bin_of(theta[g])], 1)] = g;
}

}  // namespace cnb

using namespace cnb;

extern "C" int cnb_order_buckets(const float *theta_per_bucket, const int32_t *workspace,
                                 int32_t *order, void *stream) {
    if (!theta_per_bucket || !workspace || !order) return CNB_E_INVALID_ARG;
    k_order_buckets<<<1, 1024, 0, as_stream(stream)>>>(theta_per_bucket, workspace, order);
    return launch_status();
}

extern "C" int cnb_pack_nodes(const float *n_mass, const float *n_com, const float *n_min,
                              const float *n_max, const int32_t *children, float *node_table,
                              int64_t n_nodes, void *stream) {
    if (n_nodes < 0) return CNB_E_INVALID_ARG;
    if (n_nodes == 0) return CNB_OK;
    if (!n_mass || !n_com || !n_min || !n_max || !children || !node_table)
        return CNB_E_INVALID_ARG;
    if ((reinterpret_cast<uintptr_t>(node_table) & 15) || (reinterpret_cast<uintptr_t>(children) & 7))
        return CNB_E_INVALID_ARG;
    float4 *rec = reinterpret_cast<float4 *>(node_table);
    k_pack_nodes<<<grid_for(n_nodes, 256), 256, 0, as_stream(stream)>>>(
        n_mass, n_com, n_min, n_max, reinterpret_cast<const int2 *>(children), rec,
        rec + 2 * n_nodes, n_nodes);
    return launch_status();
}

template <int BPL, int WARPS, int LAW, int STACK>
static int launch_shape(GroupedParams &P, cudaStream_t st) {
    const size_t smem = grouped_smem<BPL, LAW != 0>(WARPS, STACK);
    CNB_CUDA(cudaFuncSetAttribute(k_forces_grouped<BPL, WARPS, LAW, STACK>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_forces_grouped<BPL, WARPS, LAW, STACK>,
                                                  WARPS * 32, smem);
    // persistent grid: the work counter hands out buckets
    k_forces_grouped<BPL, WARPS, LAW, STACK>
        <<<kSMs * (per_sm > 0 ? per_sm : 1), WARPS * 32, smem, st>>>(P);
    return launch_status();
}

template <int BPL, int WARPS>
static int launch_law(GroupedParams &P, cudaStream_t st) {
    if (P.mac == CNB_MAC_PERIODIC) return launch_shape<BPL, WARPS, 0, kGStackPeriodic>(P, st);
    if (P.mac != CNB_MAC_EWALD) return launch_shape<BPL, WARPS, 0, kGStack>(P, st);
    return P.quad ? launch_shape<BPL, WARPS, 2, kGStack>(P, st)
                  : launch_shape<BPL, WARPS, 1, kGStack>(P, st);
}

static int launch_grouped(GroupedParams &P, int bodies_per_lane, int block_warps,
                          cudaStream_t st) {
    CNB_CUDA(cudaMemsetAsync(P.ws + 1, 0, 2 * sizeof(int32_t), st));
    if (P.mac == CNB_MAC_REF_X) return launch_exact(P, bodies_per_lane, block_warps, st);
    switch (bodies_per_lane * 16 + block_warps) {
        case 16 + 2: return launch_law<1, 2>(P, st);
        case 16 + 4: return launch_law<1, 4>(P, st);
        case 16 + 8: return launch_law<1, 8>(P, st);
        case 32 + 2: return launch_law<2, 2>(P, st);
        case 32 + 4: return launch_law<2, 4>(P, st);
        case 32 + 8: return launch_law<2, 8>(P, st);
        default: return CNB_E_INVALID_ARG;
    }
}

static int grouped_common(GroupedParams &P, const float *px, const float *py, const float *pz,
                          const float *node_table, int32_t *workspace, float *force, int64_t n,
                          const float *theta_per_bucket, int mac, int bodies_per_lane,
                          int block_warps, double G, unsigned long long *stats, int32_t *status) {
    if (n < 0 || (mac != CNB_MAC_REF_X && mac != CNB_MAC_REF_X_BUCKET && mac != CNB_MAC_PERIODIC))
        return CNB_E_INVALID_ARG;
    if (bodies_per_lane != 1 && bodies_per_lane != 2) return CNB_E_INVALID_ARG;
    if (block_warps != 2 && block_warps != 4 && block_warps != 8) return CNB_E_INVALID_ARG;
    if (n == 0) return CNB_OK;
    if (!px || !py || !pz || !node_table || !force || !workspace) return CNB_E_INVALID_ARG;
    if ((reinterpret_cast<uintptr_t>(node_table) & 15) || (reinterpret_cast<uintptr_t>(workspace) & 15))
        return CNB_E_INVALID_ARG;
    if (2 * n - 1 > (int64_t)INT32_MAX) return CNB_E_TOO_LARGE;
    const int64_t m = 2 * n - 1;
    P = GroupedParams{};
    P.px = px;
    P.py = py;
    P.pz = pz;
    P.rec = reinterpret_cast<const float4 *>(node_table);
    P.aabb = P.rec + 2 * m;
    P.force = force;
    P.ws = workspace;
    P.buckets = reinterpret_cast<const int4 *>(workspace + 4);
    P.theta_per_bucket = theta_per_bucket;
    P.G = (float)G;
    P.box = 1.0f;
    P.mac = mac;
    P.n = n;
    P.m_nodes = m;
    P.root = n > 1 ? (int32_t)n : 0;
    P.stats = stats;
    P.status = status;
    return CNB_OK;
}

extern "C" int cnb_forces_grouped(const float *px, const float *py, const float *pz,
                                  const float *node_table, int32_t *workspace, float *force,
                                  int64_t n, double theta, const float *theta_per_bucket,
                                  int mac, int bodies_per_lane, int block_warps, double G,
                                  double soft, double box, double slab_mass,
                                  unsigned long long *stats, int32_t *status, void *stream) {
    GroupedParams P;
    CNB_TRY(grouped_common(P, px, py, pz, node_table, workspace, force, n, theta_per_bucket, mac,
                           bodies_per_lane, block_warps, G, stats, status));
    if (n == 0) return CNB_OK;
    P.theta = (float)theta;
    P.theta_sq = theta * theta;
    P.soft2 = (float)(soft * soft);
    P.box = (float)box;
    P.slab_mass = (float)slab_mass;
    return launch_grouped(P, bodies_per_lane, block_warps, as_stream(stream));
}

// Two-level workspace (bytes from offset 0, each part 16-byte aligned):
//   16 B header | supers int4[n] | hdr int4[L] | super_of_body int32[n] |
//   near int32[L * near_cap] | far float4[L * far_cap]
// with L the number of super-bucket list slots the given size holds.
static constexpr int kFarCap = 2048, kNearCap = 256;

static int64_t align16(int64_t b) { return (b + 15) & ~(int64_t)15; }

static int64_t two_level_fixed_bytes(int64_t n) {
    return 16 + 16 * n + align16(4 * n);
}

static int64_t two_level_slot_bytes() {
    return 16 + 4LL * kNearCap + 16LL * kFarCap;
}

extern "C" int64_t cnb_two_level_workspace_bytes(int64_t n, int super_bodies) {
    if (n < 0 || super_bodies < 32) return -1;
    // super-buckets average well over a quarter of the limit; the rest walk from the root
    int64_t slots = 4 * n / super_bodies + 64;
    if (slots > n) slots = n > 0 ? n : 1;
    return two_level_fixed_bytes(n) + slots * two_level_slot_bytes();
}

extern "C" int cnb_forces_two_level(const float *px, const float *py, const float *pz,
                                    const float *node_table, const int32_t *ranges,
                                    const int32_t *parents, int32_t *workspace,
                                    void *super_ws, int64_t super_ws_bytes, int super_bodies,
                                    float *force, int64_t n, double theta, int mac,
                                    int bodies_per_lane, int block_warps, double G, double soft,
                                    double box, unsigned long long *stats, int32_t *status,
                                    void *stream) {
    if (mac != CNB_MAC_REF_X && mac != CNB_MAC_REF_X_BUCKET) return CNB_E_INVALID_ARG;
    GroupedParams P;
    CNB_TRY(grouped_common(P, px, py, pz, node_table, workspace, force, n, nullptr, mac,
                           bodies_per_lane, block_warps, G, stats, status));
    if (n == 0) return CNB_OK;
    // NULL ranges and parents: super_ws already holds this tree's super-bucket table
    const bool table_built = !ranges && !parents;
    if (!super_ws || (reinterpret_cast<uintptr_t>(super_ws) & 15) || super_bodies < 32 ||
        (n > 1 && !table_built && (!ranges || !parents)))
        return CNB_E_INVALID_ARG;
    const int64_t fixed = two_level_fixed_bytes(n);
    if (super_ws_bytes < fixed + two_level_slot_bytes()) return CNB_E_INVALID_ARG;
    int64_t slots = (super_ws_bytes - fixed) / two_level_slot_bytes();
    if (slots > n) slots = n;
    if (slots > INT32_MAX) slots = INT32_MAX;
    cudaStream_t st = as_stream(stream);
    P.theta = (float)theta;
    P.theta_sq = theta * theta;
    P.soft2 = (float)(soft * soft);
    P.box = (float)box;

    unsigned char *base = static_cast<unsigned char *>(super_ws);
    int32_t *sws = reinterpret_cast<int32_t *>(base);
    const int4 *supers = reinterpret_cast<const int4 *>(base + 16);
    int4 *hdr = reinterpret_cast<int4 *>(base + 16 + 16 * n);
    int32_t *super_of_body = reinterpret_cast<int32_t *>(base + 16 + 16 * n + 16 * slots);
    int32_t *near = reinterpret_cast<int32_t *>(base + 16 + 16 * n + 16 * slots + align16(4 * n));
    float4 *far = reinterpret_cast<float4 *>(reinterpret_cast<unsigned char *>(near) +
                                             4LL * kNearCap * slots);
    if (!table_built) CNB_TRY(cnb_make_buckets(ranges, parents, n, super_bodies, sws, stream));

    SuperParams S{};
    S.rec = P.rec;
    S.aabb = P.aabb;
    S.sws = sws;
    S.supers = supers;
    S.hdr = hdr;
    S.super_of_body = super_of_body;
    S.far = far;
    S.near = near;
    S.far_cap = kFarCap;
    S.near_cap = kNearCap;
    S.max_listed = (int)slots;
    S.th2 = (float)(theta * theta);
    S.box = P.box;
    S.half_box = 0.5f * P.box;
    S.m_nodes = P.m_nodes;
    S.root = P.root;
    S.stats = stats;
    S.status = status;
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_super_lists, kSWarps * 32, 0);
    k_super_lists<<<kSMs * (per_sm > 0 ? per_sm : 1), kSWarps * 32, 0, st>>>(S);
    CNB_TRY(launch_status());

    P.super_of_body = super_of_body;
    P.super_hdr = hdr;
    P.far_lists = far;
    P.near_lists = near;
    P.far_cap = kFarCap;
    P.near_cap = kNearCap;
    return launch_grouped(P, bodies_per_lane, block_warps, st);
}

extern "C" int cnb_forces_grouped_ewald(const float *px, const float *py, const float *pz,
                                        const float *node_table, int32_t *workspace, float *force,
                                        int64_t n, double theta, const float *theta_per_bucket,
                                        int bodies_per_lane, int block_warps, double G, double soft,
                                        const float *ewald_table, int ewald_nt,
                                        const float *quad, const int32_t *bucket_order,
                                        int32_t *bucket_inter, unsigned long long *stats,
                                        int32_t *status, void *stream) {
    GroupedParams P;
    CNB_TRY(grouped_common(P, px, py, pz, node_table, workspace, force, n, theta_per_bucket,
                           CNB_MAC_REF_X, bodies_per_lane, block_warps, G, stats, status));
    if (n == 0) return CNB_OK;
    if (!ewald_table || ewald_nt < 2 || ewald_nt > 512 ||
        (reinterpret_cast<uintptr_t>(ewald_table) & 15))
        return CNB_E_INVALID_ARG;
    P.mac = CNB_MAC_EWALD;
    P.theta = (float)theta;
    P.theta_sq = theta * theta;
    P.soft2 = (float)(soft * soft);
    P.box = 1.0f;
    P.ewald = reinterpret_cast<const float4 *>(ewald_table);
    P.ewald_nt = ewald_nt;
    if (quad && (reinterpret_cast<uintptr_t>(quad) & 15)) return CNB_E_INVALID_ARG;
    P.quad = reinterpret_cast<const float4 *>(quad);
    P.bucket_order = bucket_order;
    P.bucket_inter = bucket_inter;
    return launch_grouped(P, bodies_per_lane, block_warps, as_stream(stream));
}

extern "C" int cnb_forces_grouped_boxes_ewald(const float *px, const float *py, const float *pz,
                                              const float *node_table, int32_t *workspace,
                                              float *force, int64_t n, const uint64_t *codes,
                                              int box_bits, const int32_t *box_roots,
                                              const float *box_params,
                                              const float *theta_per_bucket, int bodies_per_lane,
                                              int block_warps, double G, const float *ewald_table,
                                              int ewald_nt, int32_t *bucket_inter,
                                              unsigned long long *stats, int32_t *status,
                                              void *stream) {
    GroupedParams P;
    CNB_TRY(grouped_common(P, px, py, pz, node_table, workspace, force, n, theta_per_bucket,
                           CNB_MAC_REF_X, bodies_per_lane, block_warps, G, stats, status));
    if (n == 0) return CNB_OK;
    if (!codes || !box_roots || !box_params || box_bits < 0 || box_bits > 30)
        return CNB_E_INVALID_ARG;
    if (!ewald_table || ewald_nt < 2 || ewald_nt > 512 ||
        (reinterpret_cast<uintptr_t>(ewald_table) & 15) ||
        (reinterpret_cast<uintptr_t>(box_params) & 15))
        return CNB_E_INVALID_ARG;
    P.mac = CNB_MAC_EWALD;
    P.codes = codes;
    P.box_shift = 3 * ((63 - box_bits) / 3);
    P.box_roots = box_roots;
    P.box_params = reinterpret_cast<const float4 *>(box_params);
    P.ewald = reinterpret_cast<const float4 *>(ewald_table);
    P.ewald_nt = ewald_nt;
    P.bucket_inter = bucket_inter;
    return launch_grouped(P, bodies_per_lane, block_warps, as_stream(stream));
}

extern "C" int cnb_forces_grouped_boxes(const float *px, const float *py, const float *pz,
                                        const float *node_table, int32_t *workspace, float *force,
                                        int64_t n, const uint64_t *codes, int box_bits,
                                        const int32_t *box_roots, const float *box_params,
                                        const float *theta_per_bucket, int mac,
                                        int bodies_per_lane, int block_warps, double G,
                                        unsigned long long *stats, int32_t *status,
                                        void *stream) {
    GroupedParams P;
    CNB_TRY(grouped_common(P, px, py, pz, node_table, workspace, force, n, theta_per_bucket, mac,
                           bodies_per_lane, block_warps, G, stats, status));
    if (n == 0) return CNB_OK;
    if (!codes || !box_roots || !box_params || box_bits < 0 || box_bits > 30)
        return CNB_E_INVALID_ARG;
    if (reinterpret_cast<uintptr_t>(box_params) & 15) return CNB_E_INVALID_ARG;
    P.codes = codes;
    P.box_shift = 3 * ((63 - box_bits) / 3);
    P.box_roots = box_roots;
    P.box_params = reinterpret_cast<const float4 *>(box_params);
    return launch_grouped(P, bodies_per_lane, block_warps, as_stream(stream));
}
