// forces_exact.cu -- the warp-per-bucket traversal with the reference's own
// opening decisions (src/kernels/physics_kernels.py:14-153, opening test
// :131-136): every body receives exactly the nodes its per-body stack walk
// accepts, in float32 arithmetic.
//
// One warp takes a bucket (a maximal subtree of at most 32*BPL bodies, lane l
// holding bodies l and l + 32).  Stack entries carry the set of the bucket's
// bodies that reached the node (a 64-bit mask: bit l of word b is body
// l + 32b); entries reached by the whole bucket sit on the main stack as
// plain node indices, the others on a second stack with their mask.  Each
// lane classifies one node against the bucket's box with the reference's
// test, sx^2 < theta^2 d^2 (sx the node's x-extent, set to the box above
// half a box; d the minimum-image distance from the body to the node's CoM):
//   every body of the mask accepts it   (sx^2 < theta^2 dmin^2)  -> list entry
//   every body of the mask opens it     (sx^2 > theta^2 dmax^2)  -> push children
//   the box cannot tell                                          -> per-body item
// with dmin / dmax the smallest / largest distance any point of the box can
// have to the CoM, widened by kBoxSlack and compared with a relative margin
// so that float32 rounding never decides.  Per-body items are evaluated by
// all lanes (each body its own d^2 and test, the force of the bodies that
// accept applied at once); the bodies that open the node push its children
// with their mask.  Leaves are accepted by every body that reaches them.
//
// Per body the float32 test reproduces the reference's float64 decision:
// the CoM difference fl32(c - x) is the reference's own float32 value, its
// minimum image d - rint(d) is exact in float32, and where the float32
// d^2 leaves sx^2 and theta^2 d^2 within kRelMargin of each other (or d^2
// within a band around the cut 1e-7) the test is redone in float64 like the
// reference.  The forces differ from the reference's only by float32 against
// float64 arithmetic and summation order.
//
// Lists: entries with one image for every body of the bucket and out of the
// cut's reach go to the whole-bucket list (applied as in forces_grouped.cu:
// packed float2 for two bodies per lane, no image, no cut) or, reached by part
// of the bucket, to the masked list (the same, the mass selected per body by
// the entry's mask); every other accepted entry keeps the node's raw CoM and
// is applied with the per-pair minimum image, the cut and its mask.
// Per-body items carry the band [lo, hi] around s^2 / theta^2 inside which
// the float32 d^2 cannot decide, and flags for the per-pair image and the
// cut, so the common item is a handful of packed operations per body pair;
// lane j keeps item j's mask of opening bodies and the children of a round's
// items are pushed together after them.
//
// The node stacks live in shared memory (see kXWords); a bucket that would
// outgrow them in the main pass is walked again by a second launch with a
// larger region, so deep walks keep their exact node sets.
//
// Limit: the reference's 64-entry stack drops children when full
// (physics_kernels.py:143-149).  That happens only for trees deeper than
// about 63 levels; the exact walk has no such drop.
#include "grouped.cuh"

namespace cnb {

constexpr float kCutLo = 0.99999e-7f, kCutHi = 1.00001e-7f;  // float64 band around the cut

// The two node stacks of a warp share one region of XW words: entries
// reached by the whole bucket (one word, the node) grow up from word 0,
// entries reached by part of it (three words: node, mask low, mask high)
// grow down from the end.  The main pass gives up on a bucket whose stacks
// would meet (it marks the bucket's record and writes no force for it); a
// second pass walks only those buckets again with a region of
// kXWordsRedo words, and a push that would overflow that one drops the
// children and flags CNB_FLAG_LIST_OVERFLOW.  The deepest use measured at
// theta = 0.5 on 128^3 and 256^3 Zel'dovich and evolved states (two-level
// walk included) is 568 words; 864 is the most that keeps ten 2-warp
// blocks (20 warps) per SM; smaller angles walk deeper and start wider.
constexpr int kXWords = 864;       // main pass, theta >= 0.4
constexpr int kXWordsWide = 2048;  // main pass, theta < 0.4
constexpr int kXWordsRedo = 4096;  // the buckets a main pass gave up on
template <int XW> __device__ __forceinline__ int part_word(int k) { return XW - 3 * (k + 1); }

// per-warp shared memory: the whole-bucket and masked lists (packed for two
// bodies per lane), the per-pair list (one float4 per entry), the per-body
// items of one round, the two lists' masks and the stack region
template <int BPL> __host__ __device__ constexpr int exact_f4_per_warp() {
    return 2 * kGList * entry_width<BPL>() + kGList + 3 * 32;
}
constexpr int kExactMasksPerWarp = 2 * kGList;  // uint2

template <int BPL>
constexpr size_t exact_smem(int warps, int xw) {
    return (size_t)warps * (exact_f4_per_warp<BPL>() * sizeof(float4) +
                            kExactMasksPerWarp * sizeof(uint2) + xw * sizeof(int32_t));
}

// per-body item flags
constexpr int kItemWrap = 1;  // the CoM's minimum image can differ between the bucket's bodies
constexpr int kItemNear = 2;  // the item is close enough to the bucket for the cut to apply

__device__ __forceinline__ float2 dup2(float a) { return make_float2(a, a); }

// d - rint(d) through the 1.5 * 2^23 rounding constant (|d| < 2^22): the
// reference's d - round(d), exact in float32 for |d| < 1
__device__ __forceinline__ float minus_image(float d) {
    return d - __fsub_rn(__fadd_rn(d, 12582912.f), 12582912.f);
}
__device__ __forceinline__ float2 minus_image2(float2 d) {
    const float2 rc = dup2(12582912.f), nrc = dup2(-12582912.f);
    return __ffma2_rn(__fadd2_rn(__fadd2_rn(d, rc), nrc), dup2(-1.f), d);
}

// The reference's test for one body, sx^2 < theta^2 d^2, in float64: called
// only when the float32 d^2 lies within the margin band of s^2 / theta^2.
__device__ __noinline__ bool ref_accepts_f64(float s, double th2d, float dx, float dy, float dz) {
    const double d2d = (double)dx * dx + (double)dy * dy + (double)dz * dz;
    return (double)s * (double)s < th2d * d2d;
}

// The reference's cut d^2 > 1e-7 (float64), float32 outside a narrow band.
__device__ __forceinline__ bool ref_outside_cut(float dx, float dy, float dz, float d2) {
    if (d2 > kCutHi) return true;
    if (d2 < kCutLo) return false;
    const double d2d = (double)dx * dx + (double)dy * dy + (double)dz * dz;
    return d2d > 1e-7;
}

// Entry j of a list as the two packed float4 (x, x, y, y), (z, z, m, m) of the
// two-bodies-per-lane loop: stored so (put_entry), or SINGLE: stored once as
// (x, y, z, m) and duplicated here (the rarely filled per-pair list).
template <bool SINGLE>
__device__ __forceinline__ void entry_pair(const float4 *list, int j, float4 &a, float4 &b) {
    if (SINGLE) {
        const float4 e = list[j];
        a = make_float4(e.x, e.x, e.y, e.y);
        b = make_float4(e.z, e.z, e.w, e.w);
    } else {
        a = list[2 * j];
        b = list[2 * j + 1];
    }
}

// Masked list: cnt entries applied to the lane's bodies in the entry's mask.
// WRAP_CUT: raw CoM, one float4 per entry, with the per-pair minimum image
// and the cut; otherwise the CoM at the one image every body of the bucket
// sees, out of the cut's reach (two float4 per entry for two bodies per
// lane, as put_entry writes them).
template <int BPL, bool WRAP_CUT>
__device__ __forceinline__ void apply_masked(const float4 *list, const uint2 *masks, int cnt,
                                             int lane, const float (&x)[BPL], const float (&y)[BPL],
                                             const float (&z)[BPL], float soft2, float (&ax)[BPL],
                                             float (&ay)[BPL], float (&az)[BPL]) {
    const float cut = soft2 + 1e-7f;
    if constexpr (BPL == 2) {
        const float2 nx = make_float2(-x[0], -x[1]), ny = make_float2(-y[0], -y[1]),
                     nz = make_float2(-z[0], -z[1]);
        const float2 s2 = dup2(soft2);
        float2 fx = make_float2(ax[0], ax[1]), fy = make_float2(ay[0], ay[1]),
               fz = make_float2(az[0], az[1]);
        // eight entries at a time: loads, distances and masses first, then the
        // inverse cubes and the accumulation in list order
        int j = 0;
        for (; j + 8 <= cnt; j += 8) {
            float2 dx[8], dy[8], dz[8], w[8], q[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                float4 a, b;
                entry_pair<WRAP_CUT>(list, j + u, a, b);
                const uint2 mk = masks[j + u];
                dx[u] = __fadd2_rn(make_float2(a.x, a.y), nx);
                dy[u] = __fadd2_rn(make_float2(a.z, a.w), ny);
                dz[u] = __fadd2_rn(make_float2(b.x, b.y), nz);
                if (WRAP_CUT) {
                    dx[u] = minus_image2(dx[u]);
                    dy[u] = minus_image2(dy[u]);
                    dz[u] = minus_image2(dz[u]);
                }
                q[u] = __ffma2_rn(dx[u], dx[u], __ffma2_rn(dy[u], dy[u], __ffma2_rn(dz[u], dz[u], s2)));
                const bool u0 = (mk.x >> lane) & 1u, u1 = (mk.y >> lane) & 1u;
                w[u] = make_float2(u0 && (!WRAP_CUT || q[u].x > cut) ? b.z : 0.f,
                                   u1 && (!WRAP_CUT || q[u].y > cut) ? b.w : 0.f);
            }
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const float2 r = make_float2(rsqrtf(q[u].x), rsqrtf(q[u].y));
                const float2 f = __fmul2_rn(__fmul2_rn(__fmul2_rn(w[u], r), r), r);
                fx = __ffma2_rn(f, dx[u], fx);
                fy = __ffma2_rn(f, dy[u], fy);
                fz = __ffma2_rn(f, dz[u], fz);
            }
        }
        for (; j < cnt; ++j) {
            float4 a, b;
            entry_pair<WRAP_CUT>(list, j, a, b);
            const uint2 mk = masks[j];
            float2 dx = __fadd2_rn(make_float2(a.x, a.y), nx);
            float2 dy = __fadd2_rn(make_float2(a.z, a.w), ny);
            float2 dz = __fadd2_rn(make_float2(b.x, b.y), nz);
            if (WRAP_CUT) {
                dx = minus_image2(dx);
                dy = minus_image2(dy);
                dz = minus_image2(dz);
            }
            const float2 q = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __ffma2_rn(dz, dz, s2)));
            const bool u0 = (mk.x >> lane) & 1u, u1 = (mk.y >> lane) & 1u;
            const float2 w = make_float2(u0 && (!WRAP_CUT || q.x > cut) ? b.z : 0.f,
                                         u1 && (!WRAP_CUT || q.y > cut) ? b.w : 0.f);
            const float2 r = make_float2(rsqrtf(q.x), rsqrtf(q.y));
            const float2 f = __fmul2_rn(__fmul2_rn(__fmul2_rn(w, r), r), r);
            fx = __ffma2_rn(f, dx, fx);
            fy = __ffma2_rn(f, dy, fy);
            fz = __ffma2_rn(f, dz, fz);
        }
        ax[0] = fx.x; ax[1] = fx.y;
        ay[0] = fy.x; ay[1] = fy.y;
        az[0] = fz.x; az[1] = fz.y;
    } else {
#pragma unroll 4
        for (int j = 0; j < cnt; ++j) {
            const float4 e = list[j];
            const bool u = (masks[j].x >> lane) & 1u;
#pragma unroll
            for (int b = 0; b < BPL; ++b) {
                float dx = e.x - x[b], dy = e.y - y[b], dz = e.z - z[b];
                if (WRAP_CUT) {
                    dx = minus_image(dx);
                    dy = minus_image(dy);
                    dz = minus_image(dz);
                }
                const float q = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, soft2)));
                const float r = rsqrtf(q);
                const float f = (u && (!WRAP_CUT || q > cut)) ? e.w * r * r * r : 0.f;
                ax[b] = fmaf(f, dx, ax[b]);
                ay[b] = fmaf(f, dy, ay[b]);
                az[b] = fmaf(f, dz, az[b]);
            }
        }
    }
}

// One per-body item for the lane's bodies: I = raw CoM and mass, J = (s,
// lo, hi, flags) with [lo, hi] the float32 band around s^2 / theta^2 where
// float64 decides, bodies in (m0, m1).  Adds the force of the bodies that
// accept; returns which of them open the node.
template <int BPL>
__device__ __forceinline__ void per_body_item(float4 I, float4 J, uint32_t m0, uint32_t m1, int lane,
                                              double th2d, float soft2, const float (&x)[BPL],
                                              const float (&y)[BPL], const float (&z)[BPL],
                                              float (&ax)[BPL], float (&ay)[BPL], float (&az)[BPL],
                                              bool (&opn)[BPL]) {
    const int flags = __float_as_int(J.w);
    if constexpr (BPL == 2) {
        float2 dx = __fadd2_rn(dup2(I.x), make_float2(-x[0], -x[1]));
        float2 dy = __fadd2_rn(dup2(I.y), make_float2(-y[0], -y[1]));
        float2 dz = __fadd2_rn(dup2(I.z), make_float2(-z[0], -z[1]));
        if (flags & kItemWrap) {
            dx = minus_image2(dx);
            dy = minus_image2(dy);
            dz = minus_image2(dz);
        }
        const float2 d2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
        bool a0 = d2.x > J.z, a1 = d2.y > J.z;
        const bool in0 = (m0 >> lane) & 1u, in1 = (m1 >> lane) & 1u;
        if (in0 && !a0 && !(d2.x < J.y)) a0 = ref_accepts_f64(J.x, th2d, dx.x, dy.x, dz.x);
        if (in1 && !a1 && !(d2.y < J.y)) a1 = ref_accepts_f64(J.x, th2d, dx.y, dy.y, dz.y);
        const bool u0 = in0 && a0, u1 = in1 && a1;
        opn[0] = in0 && !a0;
        opn[BPL - 1] = in1 && !a1;
        bool f0 = u0, f1 = u1;
        if (flags & kItemNear) {
            f0 = f0 && ref_outside_cut(dx.x, dy.x, dz.x, d2.x);
            f1 = f1 && ref_outside_cut(dx.y, dy.y, dz.y, d2.y);
        }
        // an item every reaching body opens adds no force (a third of them)
        if (!__any_sync(0xffffffffu, f0 || f1)) return;
        const float2 q = __fadd2_rn(d2, dup2(soft2));
        const float2 r = make_float2(rsqrtf(q.x), rsqrtf(q.y));
        const float2 w = make_float2(f0 ? I.w : 0.f, f1 ? I.w : 0.f);
        const float2 f = __fmul2_rn(__fmul2_rn(__fmul2_rn(w, r), r), r);
        const float2 fx = __ffma2_rn(f, dx, make_float2(ax[0], ax[1]));
        const float2 fy = __ffma2_rn(f, dy, make_float2(ay[0], ay[1]));
        const float2 fz = __ffma2_rn(f, dz, make_float2(az[0], az[1]));
        ax[0] = fx.x; ax[1] = fx.y;
        ay[0] = fy.x; ay[1] = fy.y;
        az[0] = fz.x; az[1] = fz.y;
    } else {
#pragma unroll
        for (int b = 0; b < BPL; ++b) {
            float dx = I.x - x[b], dy = I.y - y[b], dz = I.z - z[b];
            if (flags & kItemWrap) {
                dx = minus_image(dx);
                dy = minus_image(dy);
                dz = minus_image(dz);
            }
            const float d2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
            const bool in = ((b == 0 ? m0 : m1) >> lane) & 1u;
            bool a = d2 > J.z;
            if (in && !a && !(d2 < J.y)) a = ref_accepts_f64(J.x, th2d, dx, dy, dz);
            const bool u = in && a;
            opn[b] = in && !a;
            const bool fu = u && (!(flags & kItemNear) || ref_outside_cut(dx, dy, dz, d2));
            const float r = rsqrtf(d2 + soft2);
            const float f = fu ? I.w * r * r * r : 0.f;
            ax[b] = fmaf(f, dx, ax[b]);
            ay[b] = fmaf(f, dy, ay[b]);
            az[b] = fmaf(f, dz, az[b]);
        }
    }
}

// Applies the first 32 entries of a list and moves the rest to the front.
template <int BPL, int KIND>
__device__ __forceinline__ void flush32(float4 *lst, uint2 *msk, int &cnt, int lane,
                                        const float (&x)[BPL], const float (&y)[BPL],
                                        const float (&z)[BPL], float soft2, float (&ax)[BPL],
                                        float (&ay)[BPL], float (&az)[BPL]) {
    constexpr int EW = KIND == 2 ? 1 : entry_width<BPL>();  // the per-pair list: one float4
    if (KIND == 0) apply_entries<BPL, false, false>(lst, 32, x, y, z, soft2, ax, ay, az);
    else if (KIND == 1) apply_masked<BPL, false>(lst, msk, 32, lane, x, y, z, soft2, ax, ay, az);
    else apply_masked<BPL, true>(lst, msk, 32, lane, x, y, z, soft2, ax, ay, az);
    __syncwarp();
#pragma unroll
    for (int w = 0; w < EW; ++w)
        if (lane < cnt - 32) lst[EW * lane + w] = lst[EW * (32 + lane) + w];
    if (KIND != 0 && lane < cnt - 32) msk[lane] = msk[32 + lane];
    cnt -= 32;
    __syncwarp();
}

// REDO false: the main pass over every bucket (work counter); true: the
// buckets a main pass gave up on (bucket record's fourth word = 1), found by
// a strided scan of the table and cleared when done.
// Twenty warps per SM: ten 2-warp blocks fit the shared memory of the main
// pass; the register bound (at most 102 for 2 or 4 warps per block) keeps them.
template <int BPL, int WARPS, int XW, bool REDO, bool TEST = false>
__global__ void __launch_bounds__(WARPS * 32, 20 / WARPS) k_forces_exact(GroupedParams P) {
    static_assert(BPL == 1 || BPL == 2, "one or two bodies per lane");
    extern __shared__ __align__(16) unsigned char x_smem[];
    constexpr int EW = entry_width<BPL>();
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const uint32_t lt = (1u << lane) - 1u;
    float4 *f4 = reinterpret_cast<float4 *>(x_smem);
    float4 *list = f4 + wib * exact_f4_per_warp<BPL>();  // whole bucket, one image, no cut
    float4 *mlist = list + kGList * EW;                   // masked, one image, no cut
    float4 *xlist = mlist + kGList * EW;                  // per-pair image and cut, any mask
    float4 *plist = xlist + kGList;                       // per-body items (3 float4 each)
    uint2 *mbase = reinterpret_cast<uint2 *>(f4 + WARPS * exact_f4_per_warp<BPL>());
    uint2 *mmask = mbase + wib * kExactMasksPerWarp;
    uint2 *xmask = mmask + kGList;
    // the stack region: whole-bucket entries from word 0 up, (node, mask) entries from the end down
    int32_t *stack = reinterpret_cast<int32_t *>(mbase + WARPS * kExactMasksPerWarp) +
                     wib * XW;

    unsigned long long n_tests = 0, n_inter = 0, n_wrap = 0;
    int max_top = 0;
    bool overflow = false;
    const int n_buckets = P.ws[0];
    const float half_box = 0.5f * P.box;

    int4 *table = reinterpret_cast<int4 *>(P.ws + 4);  // the bucket records (P.buckets)
    // redo: this warp's share of the table, 32 records at a time (lane l reads record
    // chunk + l); marked holds the records of the chunk still to walk
    int chunk = (blockIdx.x * WARPS + wib) * 32;
    uint32_t marked = 0u;
    for (;;) {
        int g = 0;
        if (REDO) {
            while (marked == 0u && chunk < n_buckets) {
                const int r = chunk + lane;
                marked = __ballot_sync(0xffffffffu, r < n_buckets && table[r].w == 1);
                if (marked == 0u) chunk += gridDim.x * WARPS * 32;
            }
            if (marked == 0u) break;
            g = chunk + __ffs(marked) - 1;
            marked &= marked - 1u;
            if (marked == 0u) chunk += gridDim.x * WARPS * 32;
        } else {
            if (lane == 0) g = atomicAdd(P.ws + 1, 1);
            g = __shfl_sync(0xffffffffu, g, 0);
            if (g >= n_buckets) break;
            if (P.bucket_order) g = P.bucket_order[g];
        }
        const int4 bk = P.buckets[g];
        bool spill = false;  // main pass: this bucket is left to the redo pass
        uint32_t b_tests = 0, b_inter = 0, b_wrap = 0;  // this bucket's counts (lane's share)
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
        const float ghx = 0.5f * (hx - lx) + kBoxSlack, ghy = 0.5f * (hy - ly) + kBoxSlack,
                    ghz = 0.5f * (hz - lz) + kBoxSlack;
        // an entry whose image offset from the centre stays below this has one
        // minimum image for every body of the bucket
        const float wlx = 0.5f - ghx - 1e-6f, wly = 0.5f - ghy - 1e-6f, wlz = 0.5f - ghz - 1e-6f;
        // the bucket's bodies: bit l of word b is body l + 32 b
        const uint2 fm = make_uint2(count >= 32 ? 0xffffffffu : ((1u << count) - 1u),
                                    BPL == 1 || count <= 32 ? 0u
                                    : (count >= 64 ? 0xffffffffu : ((1u << (count - 32)) - 1u)));
        float th = P.theta, soft2 = P.soft2;
        double th2d = P.theta_sq;
        int32_t root = P.root;
        if (P.box_roots) {
            const uint64_t b = P.codes[bk.x] >> P.box_shift;
            const float4 bp = P.box_params[b];
            root = P.box_roots[b];
            th = bp.x;
            soft2 = bp.y * bp.y;
            th2d = (double)th * (double)th;
        }
        if (P.theta_per_bucket) {
            th = P.theta_per_bucket[g];
            th2d = (double)th * (double)th;
        }
        const float th2 = (float)th2d;
        const float inv_th2 = 1.f / th2;

        float ax[BPL], ay[BPL], az[BPL];
#pragma unroll
        for (int b = 0; b < BPL; ++b) ax[b] = ay[b] = az[b] = 0.f;
        int top = 1, ptop = 0, cnt = 0, mcnt = 0, xcnt = 0, n_acc = 0;
        bool seeded = false;
        if (P.super_of_body) {
            const int sup = P.super_of_body[bk.x];
            const int4 h = sup >= 0 ? P.super_hdr[sup] : make_int4(0, 0, 0, 0);
            if (h.w && h.z <= XW) {
                // the nodes every body of the super-bucket accepts (k_super_lists)
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
                if (lane == 0) {
                    b_inter += (uint32_t)((h.x + h.y) * count);
                    b_wrap += (uint32_t)(h.y * count);
                }
                const int32_t *near = P.near_lists + (int64_t)sup * P.near_cap;
                for (int j = lane; j < h.z; j += 32) stack[j] = near[j];
                top = h.z;
                seeded = true;
            }
        }
        if (!seeded && lane == 0) stack[0] = root;
        __syncwarp();
        int64_t rounds = 0;
        while ((top > 0 || ptop > 0) && !spill) {
            // a valid tree pushes every node at most once per bucket
            if (++rounds > P.m_nodes) {
                if (lane == 0) set_flag(P.status, CNB_FLAG_BAD_TOPOLOGY);
                break;
            }
            // part-bucket entries first (they keep the second stack short)
            const int k1 = ptop < 32 ? ptop : 32;
            const int k2 = min(top, 32 - k1);
            ptop -= k1;
            top -= k2;
            int32_t node = -1;
            uint2 mk = fm;
            if (lane < k1) {
                const int pw = part_word<XW>(ptop + lane);
                node = stack[pw];
                mk = make_uint2((uint32_t)stack[pw + 1], (uint32_t)stack[pw + 2]);
            } else if (lane < k1 + k2) {
                node = stack[top + lane - k1];
            }
            __syncwarp();
            if (node >= P.m_nodes) {
                set_flag(P.status, CNB_FLAG_BAD_TOPOLOGY);
                node = -1;
            }
            const bool whole = mk.x == fm.x && mk.y == fm.y;
            // 1: accepted by every body of the mask, 2: opened by every one, 3: per body
            int cls = 0;
            bool one_image = false, zero_image = false, near_box = false;
            float4 A = make_float4(0.f, 0.f, 0.f, 0.f), E = A;
            float s = 0.f;
            int32_t c0 = -1, c1 = -1;
            if (node >= 0) {
                A = __ldg(P.rec + 2 * node);
                const float4 S = __ldg(P.rec + 2 * node + 1);
                if (A.w > 0.f) {  // physics_kernels.py:114 (nm <= 0: skipped)
                    c0 = __float_as_int(S.z);
                    c1 = __float_as_int(S.w);
                    const float dx = A.x - gcx, dy = A.y - gcy, dz = A.z - gcz;
                    const float sx_ = image_of(dx), sy_ = image_of(dy), sz_ = image_of(dz);
                    const float adx = fabsf(dx - sx_), ady = fabsf(dy - sy_), adz = fabsf(dz - sz_);
                    const float tx = fmaxf(adx - ghx, 0.f), ty = fmaxf(ady - ghy, 0.f),
                                tz = fmaxf(adz - ghz, 0.f);
                    const float d2min = tx * tx + ty * ty + tz * tz;
                    s = S.x > half_box ? P.box : S.x;  // physics_kernels.py:131-132
                    if (c0 == -1) {
                        cls = 1;  // a leaf: used by every body that reaches it
                    } else {
                        const float ux = fminf(adx + ghx, half_box), uy = fminf(ady + ghy, half_box),
                                    uz = fminf(adz + ghz, half_box);
                        const float d2max = ux * ux + uy * uy + uz * uz;
                        const float s2 = s * s;
                        if (s2 < th2 * d2min * (1.f - kRelMargin)) cls = 1;
                        else if (s2 > th2 * d2max * (1.f + kRelMargin)) cls = 2;
                        else cls = 3;
                    }
                    near_box = d2min <= kCutGuard;
                    one_image = adx < wlx && ady < wly && adz < wlz;
                    zero_image = one_image && sx_ == 0.f && sy_ == 0.f && sz_ == 0.f;
                    E = make_float4(A.x - sx_, A.y - sy_, A.z - sz_, A.w);
                }
            }
            b_tests += (node >= 0);
            const bool to_list = cls == 1 && whole && one_image && !near_box;
            const bool to_m = cls == 1 && !whole && one_image && !near_box;
            const bool to_x = cls == 1 && !(one_image && !near_box);
            const uint32_t m_one = __ballot_sync(0xffffffffu, to_list);
            const uint32_t m_msk = __ballot_sync(0xffffffffu, to_m);
            const uint32_t m_x = __ballot_sync(0xffffffffu, to_x);
            const uint32_t m_ow = __ballot_sync(0xffffffffu, cls == 2 && whole);
            const uint32_t m_op = __ballot_sync(0xffffffffu, cls == 2 && !whole);
            const uint32_t m_pb = __ballot_sync(0xffffffffu, cls == 3);
            if (cls == 1) {
                const int nb = __popc(mk.x) + __popc(mk.y);
                b_inter += nb;
                if (to_list) {
                    put_entry<BPL>(list, cnt + __popc(m_one & lt), E);
                } else if (to_m) {
                    const int w = mcnt + __popc(m_msk & lt);
                    put_entry<BPL>(mlist, w, E);
                    mmask[w] = mk;
                } else {
                    const int w = xcnt + __popc(m_x & lt);
                    xlist[w] = A;
                    xmask[w] = mk;
                    b_wrap += nb;
                }
            }
            cnt += __popc(m_one);
            mcnt += __popc(m_msk);
            xcnt += __popc(m_x);
            const int n_ow = __popc(m_ow), n_op = __popc(m_op);
            if (top + 2 * n_ow + 3 * (ptop + 2 * n_op) > XW) {
                if (REDO) overflow = true;  // children dropped (flagged)
                else spill = true;          // the redo pass walks this bucket again
            } else {
                if (cls == 2 && whole) {
                    const int pos = top + 2 * __popc(m_ow & lt);
                    stack[pos] = c1;
                    stack[pos + 1] = c0;
                }
                if (cls == 2 && !whole) {
                    const int pos = ptop + 2 * __popc(m_op & lt);
                    const int w1 = part_word<XW>(pos), w0 = part_word<XW>(pos + 1);
                    stack[w1] = c1;
                    stack[w1 + 1] = (int32_t)mk.x;
                    stack[w1 + 2] = (int32_t)mk.y;
                    stack[w0] = c0;
                    stack[w0 + 1] = (int32_t)mk.x;
                    stack[w0 + 2] = (int32_t)mk.y;
                }
                top += 2 * n_ow;
                ptop += 2 * n_op;
            }
            const int pcnt = __popc(m_pb);
            if (cls == 3) {
                // the band [lo, hi] around s^2 / theta^2 inside which float64 decides
                const float R = s * s * inv_th2;
                const int fl = (zero_image ? 0 : kItemWrap) | (near_box ? kItemNear : 0);
                const int w = __popc(m_pb & lt);
                plist[3 * w] = A;
                plist[3 * w + 1] = make_float4(s, R * (1.f - kRelMargin), R * (1.f + kRelMargin),
                                               __int_as_float(fl));
                plist[3 * w + 2] = make_float4(__int_as_float(c0), __int_as_float(c1),
                                               __uint_as_float(mk.x), __uint_as_float(mk.y));
            }
            __syncwarp();
            // per-body items: every body of the mask decides for itself; lane j
            // keeps item j's mask of opening bodies, and the children of every
            // item that some body opened are pushed together afterwards
            uint2 my_om = make_uint2(0u, 0u);
#pragma unroll 1
            for (int j = 0; j < pcnt; ++j) {
                const float4 I = plist[3 * j], J = plist[3 * j + 1], K = plist[3 * j + 2];
                bool opn[BPL];
                per_body_item<BPL>(I, J, __float_as_uint(K.z), __float_as_uint(K.w), lane, th2d, soft2,
                                   x, y, z, ax, ay, az, opn);
                const uint32_t o0 = __ballot_sync(0xffffffffu, opn[0]);
                const uint32_t o1 = BPL == 2 ? __ballot_sync(0xffffffffu, opn[BPL - 1]) : 0u;
                if (lane == j) my_om = make_uint2(o0, o1);
            }
            if (pcnt > 0) {
                bool has = false, whole_o = false;
                int32_t k0 = -1, k1c = -1;
                if (lane < pcnt) {
                    const float4 K = plist[3 * lane + 2];
                    k0 = __float_as_int(K.x);
                    k1c = __float_as_int(K.y);
                    has = (my_om.x | my_om.y) != 0u;
                    whole_o = my_om.x == fm.x && my_om.y == fm.y;
                    // the bodies of the item's mask that did not open it accepted it
                    n_acc += __popc(__float_as_uint(K.z)) + __popc(__float_as_uint(K.w)) -
                             __popc(my_om.x) - __popc(my_om.y);
                }
                const uint32_t mw = __ballot_sync(0xffffffffu, has && whole_o);
                const uint32_t mp = __ballot_sync(0xffffffffu, has && !whole_o);
                const int nw = __popc(mw), npart = __popc(mp);
                if (top + 2 * nw + 3 * (ptop + 2 * npart) > XW) {
                    if (REDO) overflow = true;  // children dropped (flagged)
                    else spill = true;          // the redo pass walks this bucket again
                } else {
                    if (has && whole_o) {
                        const int pos = top + 2 * __popc(mw & lt);
                        stack[pos] = k1c;
                        stack[pos + 1] = k0;
                    }
                    if (has && !whole_o) {
                        const int pos = ptop + 2 * __popc(mp & lt);
                        const int w1 = part_word<XW>(pos), w0 = part_word<XW>(pos + 1);
                        stack[w1] = k1c;
                        stack[w1 + 1] = (int32_t)my_om.x;
                        stack[w1 + 2] = (int32_t)my_om.y;
                        stack[w0] = k0;
                        stack[w0 + 1] = (int32_t)my_om.x;
                        stack[w0 + 2] = (int32_t)my_om.y;
                    }
                    top += 2 * nw;
                    ptop += 2 * npart;
                }
            }
            max_top = max(max_top, top + 3 * ptop);  // words of the stack region
            __syncwarp();
            if (cnt >= 32) flush32<BPL, 0>(list, nullptr, cnt, lane, x, y, z, soft2, ax, ay, az);
            if (mcnt >= 32) flush32<BPL, 1>(mlist, mmask, mcnt, lane, x, y, z, soft2, ax, ay, az);
            if (xcnt >= 32) flush32<BPL, 2>(xlist, xmask, xcnt, lane, x, y, z, soft2, ax, ay, az);
            // tests: give up on a bucket after its first round as an overflow would
            if (TEST && rounds == 1 && g % P.test_spill_every == 0) spill = true;
        }
        if (!REDO && spill) {
            // the stacks would meet: no force and no counts from this pass; the redo
            // pass walks it again
            if (lane == 0) table[g].w = 1;
            __syncwarp();
            continue;
        }
        apply_entries<BPL, false, false>(list, cnt, x, y, z, soft2, ax, ay, az);
        apply_masked<BPL, false>(mlist, mmask, mcnt, lane, x, y, z, soft2, ax, ay, az);
        apply_masked<BPL, true>(xlist, xmask, xcnt, lane, x, y, z, soft2, ax, ay, az);
        __syncwarp();
        if (REDO && lane == 0) table[g].w = 0;
        n_tests += b_tests;
        n_inter += b_inter + n_acc;
        n_wrap += b_wrap + n_acc;
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
    }
    if (overflow && lane == 0) set_flag(P.status, CNB_FLAG_LIST_OVERFLOW);
    if (P.stats) {
        for (int o = 16; o > 0; o >>= 1) {
            n_tests += __shfl_xor_sync(0xffffffffu, n_tests, o);
            n_inter += __shfl_xor_sync(0xffffffffu, n_inter, o);
            n_wrap += __shfl_xor_sync(0xffffffffu, n_wrap, o);
        }
        if (lane == 0) {
            atomicAdd(P.stats, n_inter);
            atomicAdd(P.stats + 1, n_tests);
            atomicAdd(P.stats + 2, n_wrap);
        }
    }
    if (lane == 0) atomicMax(P.ws + 2, max_top);
}

template <int BPL, int WARPS, int XW, bool REDO, bool TEST = false>
static int launch_exact_pass(GroupedParams &P, cudaStream_t st) {
    const size_t smem = exact_smem<BPL>(WARPS, XW);
    CNB_CUDA(cudaFuncSetAttribute(k_forces_exact<BPL, WARPS, XW, REDO, TEST>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_forces_exact<BPL, WARPS, XW, REDO, TEST>,
                                                  WARPS * 32, smem);
    // persistent grid: the work counter (main pass) or the table scan (redo) hands out buckets
    k_forces_exact<BPL, WARPS, XW, REDO, TEST>
        <<<kSMs * (per_sm > 0 ? per_sm : 1), WARPS * 32, smem, st>>>(P);
    return launch_status();
}

template <int BPL, int WARPS>
static int launch_exact_shape(GroupedParams &P, cudaStream_t st) {
    // the main pass: smaller angles walk deeper and start with the wide region
    if (P.test_spill_every > 0)  // tests: the main pass gives up on every n-th bucket
        CNB_TRY((launch_exact_pass<BPL, WARPS, kXWords, false, true>(P, st)));
    else if (P.theta < 0.4f)
        CNB_TRY((launch_exact_pass<BPL, WARPS, kXWordsWide, false>(P, st)));
    else
        CNB_TRY((launch_exact_pass<BPL, WARPS, kXWords, false>(P, st)));
    // the buckets it gave up on, if any (otherwise every warp scans its share of the
    // bucket table and returns)
    return launch_exact_pass<BPL, 2, kXWordsRedo, true>(P, st);
}

static int g_test_spill_every = 0;  // cnb_exact_test_spill

int launch_exact(GroupedParams &P, int bodies_per_lane, int block_warps, cudaStream_t st) {
    P.test_spill_every = g_test_spill_every;
    switch (bodies_per_lane * 16 + block_warps) {
        case 16 + 2: return launch_exact_shape<1, 2>(P, st);
        case 16 + 4: return launch_exact_shape<1, 4>(P, st);
        case 16 + 8: return launch_exact_shape<1, 8>(P, st);
        case 32 + 2: return launch_exact_shape<2, 2>(P, st);
        case 32 + 4: return launch_exact_shape<2, 4>(P, st);
        case 32 + 8: return launch_exact_shape<2, 8>(P, st);
        default: return CNB_E_INVALID_ARG;
    }
}

}  // namespace cnb

extern "C" int cnb_exact_test_spill(int every) {
    if (every < 0) return CNB_E_INVALID_ARG;
    cnb::g_test_spill_every = every;
    return CNB_OK;
}
