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
// Lists: entries accepted by the whole bucket with one image for all of its
// bodies and out of the cut's reach (the bulk) are applied as in
// forces_grouped.cu (packed float2 for two bodies per lane, no image, no
// cut); every other accepted entry keeps the node's raw CoM and is applied
// with the per-pair minimum image, the cut and the entry's body mask.
//
// Limit: the reference's 64-entry stack drops children when full
// (physics_kernels.py:143-149).  That happens only for trees deeper than
// about 63 levels; the exact walk has no such drop.
#include "grouped.cuh"

namespace cnb {

constexpr int kXPStack = 256;           // (node, mask) entries per warp for part of a bucket
constexpr float kCutLo = 0.99999e-7f, kCutHi = 1.00001e-7f;  // float64 band around the cut

template <int BPL> __host__ __device__ constexpr int exact_f4_per_warp() {
    // full-bucket list, masked list (kGList entries each), per-body items (32 x 2)
    return 2 * kGList * entry_width<BPL>() + 64;
}
constexpr int kExactMasksPerWarp = kGList + 32 + kXPStack;  // uint2
constexpr int kExactIntsPerWarp = kGStack + kXPStack;         // int32

template <int BPL>
constexpr size_t exact_smem(int warps) {
    return (size_t)warps * (exact_f4_per_warp<BPL>() * sizeof(float4) +
                            kExactMasksPerWarp * sizeof(uint2) + kExactIntsPerWarp * sizeof(int32_t));
}

__device__ __forceinline__ float nearest_image(float d) {
    // rint(d) through the 1.5 * 2^23 rounding constant (|d| < 2^22)
    return __fsub_rn(__fadd_rn(d, 12582912.f), 12582912.f);
}

// The reference's test for one body: sx^2 < theta^2 d^2 on float64 values.
// The float32 form decides unless the two sides are within kRelMargin.
__device__ __forceinline__ bool ref_accepts(float s, float th2, double th2d, float dx, float dy,
                                            float dz, float d2) {
    const float s2 = s * s, t = th2 * d2;
    if (fabsf(s2 - t) > kRelMargin * t) return s2 < t;
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

// Masked list: cnt entries of raw CoM and mass (two float4 per entry for two
// bodies per lane, as put_entry writes them) applied to the lane's bodies in
// the entry's mask, with the per-pair minimum image and the cut.
template <int BPL>
__device__ __forceinline__ void apply_masked(const float4 *list, const uint2 *masks, int cnt,
                                             int lane, const float (&x)[BPL], const float (&y)[BPL],
                                             const float (&z)[BPL], float soft2, float (&ax)[BPL],
                                             float (&ay)[BPL], float (&az)[BPL]) {
    const float cut = soft2 + 1e-7f;
    if constexpr (BPL == 2) {
        const float2 nx = make_float2(-x[0], -x[1]), ny = make_float2(-y[0], -y[1]),
                     nz = make_float2(-z[0], -z[1]);
        const float2 s2 = make_float2(soft2, soft2);
        const float2 rc = make_float2(12582912.f, 12582912.f), nrc = make_float2(-12582912.f, -12582912.f);
        const float2 m1 = make_float2(-1.f, -1.f);
        float2 fx = make_float2(ax[0], ax[1]), fy = make_float2(ay[0], ay[1]),
               fz = make_float2(az[0], az[1]);
#pragma unroll 4
        for (int j = 0; j < cnt; ++j) {
            const float4 a = list[2 * j], b = list[2 * j + 1];
            const uint2 mk = masks[j];
            float2 dx = __fadd2_rn(make_float2(a.x, a.y), nx);
            float2 dy = __fadd2_rn(make_float2(a.z, a.w), ny);
            float2 dz = __fadd2_rn(make_float2(b.x, b.y), nz);
            dx = __ffma2_rn(__fadd2_rn(__fadd2_rn(dx, rc), nrc), m1, dx);
            dy = __ffma2_rn(__fadd2_rn(__fadd2_rn(dy, rc), nrc), m1, dy);
            dz = __ffma2_rn(__fadd2_rn(__fadd2_rn(dz, rc), nrc), m1, dz);
            const float2 q = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __ffma2_rn(dz, dz, s2)));
            float r0 = rsqrtf(q.x), r1 = rsqrtf(q.y);
            r0 = (q.x > cut && ((mk.x >> lane) & 1u)) ? r0 : 0.f;
            r1 = (q.y > cut && ((mk.y >> lane) & 1u)) ? r1 : 0.f;
            const float2 r = make_float2(r0, r1);
            const float2 f = __fmul2_rn(__fmul2_rn(__fmul2_rn(make_float2(b.z, b.w), r), r), r);
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
            const uint32_t mw = masks[j].x;
#pragma unroll
            for (int b = 0; b < BPL; ++b) {
                float dx = e.x - x[b], dy = e.y - y[b], dz = e.z - z[b];
                dx -= pair_image(dx);
                dy -= pair_image(dy);
                dz -= pair_image(dz);
                const float q = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, soft2)));
                const float r = rsqrtf(q);
                const float f = (q > cut && ((mw >> lane) & 1u)) ? e.w * r * r * r : 0.f;
                ax[b] = fmaf(f, dx, ax[b]);
                ay[b] = fmaf(f, dy, ay[b]);
                az[b] = fmaf(f, dz, az[b]);
            }
        }
    }
}

template <int BPL, int WARPS>
__global__ void __launch_bounds__(WARPS * 32) k_forces_exact(GroupedParams P) {
    static_assert(BPL == 1 || BPL == 2, "one or two bodies per lane");
    extern __shared__ __align__(16) unsigned char x_smem[];
    constexpr int EW = entry_width<BPL>();
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const uint32_t lt = (1u << lane) - 1u;
    float4 *f4 = reinterpret_cast<float4 *>(x_smem);
    float4 *list = f4 + wib * exact_f4_per_warp<BPL>();
    float4 *mlist = list + kGList * EW;
    float4 *plist = mlist + kGList * EW;
    uint2 *mbase = reinterpret_cast<uint2 *>(f4 + WARPS * exact_f4_per_warp<BPL>());
    uint2 *mmask = mbase + wib * kExactMasksPerWarp;
    uint2 *pmask = mmask + kGList;
    uint2 *psmask = pmask + 32;
    int32_t *stack = reinterpret_cast<int32_t *>(mbase + WARPS * kExactMasksPerWarp) +
                     wib * kExactIntsPerWarp;
    int32_t *pstack = stack + kGStack;

    unsigned long long n_tests = 0, n_inter = 0, n_wrap = 0;
    int max_top = 0;
    bool overflow = false;
    const int n_buckets = P.ws[0];
    const float half_box = 0.5f * P.box;

    for (;;) {
        int g = 0;
        if (lane == 0) g = atomicAdd(P.ws + 1, 1);
        g = __shfl_sync(0xffffffffu, g, 0);
        if (g >= n_buckets) break;
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

        float ax[BPL], ay[BPL], az[BPL];
#pragma unroll
        for (int b = 0; b < BPL; ++b) ax[b] = ay[b] = az[b] = 0.f;
        int top = 1, ptop = 0, cnt = 0, mcnt = 0;
        bool seeded = false;
        if (P.super_of_body) {
            const int sup = P.super_of_body[bk.x];
            const int4 h = sup >= 0 ? P.super_hdr[sup] : make_int4(0, 0, 0, 0);
            if (h.w) {
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
                    n_inter += (unsigned long long)(h.x + h.y) * count;
                    n_wrap += (unsigned long long)h.y * count;
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
        while (top > 0 || ptop > 0) {
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
                node = pstack[ptop + lane];
                mk = psmask[ptop + lane];
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
            bool one_image = false;
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
                    one_image = whole && d2min > kCutGuard && adx < wlx && ady < wly && adz < wlz;
                    E = make_float4(A.x - sx_, A.y - sy_, A.z - sz_, A.w);
                }
            }
            n_tests += (node >= 0);
            const uint32_t m_one = __ballot_sync(0xffffffffu, cls == 1 && one_image);
            const uint32_t m_msk = __ballot_sync(0xffffffffu, cls == 1 && !one_image);
            const uint32_t m_ow = __ballot_sync(0xffffffffu, cls == 2 && whole);
            const uint32_t m_op = __ballot_sync(0xffffffffu, cls == 2 && !whole);
            const uint32_t m_pb = __ballot_sync(0xffffffffu, cls == 3);
            if (cls == 1) {
                const int nb = __popc(mk.x) + __popc(mk.y);
                n_inter += nb;
                if (one_image) {
                    put_entry<BPL>(list, cnt + __popc(m_one & lt), E);
                } else {
                    const int w = mcnt + __popc(m_msk & lt);
                    put_entry<BPL>(mlist, w, A);
                    mmask[w] = mk;
                    n_wrap += nb;
                }
            }
            cnt += __popc(m_one);
            mcnt += __popc(m_msk);
            const int n_ow = __popc(m_ow), n_op = __popc(m_op);
            if (top + 2 * n_ow > kGStack || ptop + 2 * n_op > kXPStack) {
                overflow = true;  // children dropped (flagged)
            } else {
                if (cls == 2 && whole) {
                    const int pos = top + 2 * __popc(m_ow & lt);
                    stack[pos] = c1;
                    stack[pos + 1] = c0;
                }
                if (cls == 2 && !whole) {
                    const int pos = ptop + 2 * __popc(m_op & lt);
                    pstack[pos] = c1;
                    pstack[pos + 1] = c0;
                    psmask[pos] = mk;
                    psmask[pos + 1] = mk;
                }
                top += 2 * n_ow;
                ptop += 2 * n_op;
            }
            const int pcnt = __popc(m_pb);
            if (cls == 3) {
                const int w = __popc(m_pb & lt);
                plist[2 * w] = A;
                plist[2 * w + 1] = make_float4(s, __int_as_float(c0), __int_as_float(c1), 0.f);
                pmask[w] = mk;
            }
            __syncwarp();
            // per-body items: every body of the mask decides for itself
            for (int j = 0; j < pcnt; ++j) {
                const float4 I = plist[2 * j], J = plist[2 * j + 1];
                const uint2 pm = pmask[j];
                bool opn[BPL];
#pragma unroll
                for (int b = 0; b < BPL; ++b) {
                    const bool inm = (((b == 0 ? pm.x : pm.y) >> lane) & 1u) != 0u;
                    float dx = I.x - x[b], dy = I.y - y[b], dz = I.z - z[b];
                    dx -= nearest_image(dx);
                    dy -= nearest_image(dy);
                    dz -= nearest_image(dz);
                    const float d2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                    const bool pass = ref_accepts(J.x, th2, th2d, dx, dy, dz, d2);
                    const bool use = inm && pass;
                    opn[b] = inm && !pass;
                    n_inter += use;
                    n_wrap += use;
                    const float r = rsqrtf(d2 + soft2);
                    const float f = (use && ref_outside_cut(dx, dy, dz, d2)) ? I.w * r * r * r : 0.f;
                    ax[b] = fmaf(f, dx, ax[b]);
                    ay[b] = fmaf(f, dy, ay[b]);
                    az[b] = fmaf(f, dz, az[b]);
                }
                const uint2 om = make_uint2(__ballot_sync(0xffffffffu, opn[0]),
                                            BPL == 2 ? __ballot_sync(0xffffffffu, opn[BPL - 1]) : 0u);
                if (om.x | om.y) {
                    const int32_t k0 = __float_as_int(J.y), k1c = __float_as_int(J.z);
                    if (om.x == fm.x && om.y == fm.y) {
                        if (top + 2 > kGStack) {
                            overflow = true;
                        } else {
                            if (lane == 0) {
                                stack[top] = k1c;
                                stack[top + 1] = k0;
                            }
                            top += 2;
                        }
                    } else if (ptop + 2 > kXPStack) {
                        overflow = true;
                    } else {
                        if (lane == 0) {
                            pstack[ptop] = k1c;
                            pstack[ptop + 1] = k0;
                            psmask[ptop] = om;
                            psmask[ptop + 1] = om;
                        }
                        ptop += 2;
                    }
                }
            }
            max_top = max(max_top, top + ptop);
            __syncwarp();
            if (cnt >= 32) {
                apply_entries<BPL, false, false>(list, 32, x, y, z, soft2, ax, ay, az);
                __syncwarp();
#pragma unroll
                for (int w = 0; w < EW; ++w)
                    if (lane < cnt - 32) list[EW * lane + w] = list[EW * (32 + lane) + w];
                cnt -= 32;
                __syncwarp();
            }
            if (mcnt >= 32) {
                apply_masked<BPL>(mlist, mmask, 32, lane, x, y, z, soft2, ax, ay, az);
                __syncwarp();
#pragma unroll
                for (int w = 0; w < EW; ++w)
                    if (lane < mcnt - 32) mlist[EW * lane + w] = mlist[EW * (32 + lane) + w];
                if (lane < mcnt - 32) mmask[lane] = mmask[32 + lane];
                mcnt -= 32;
                __syncwarp();
            }
        }
        apply_entries<BPL, false, false>(list, cnt, x, y, z, soft2, ax, ay, az);
        apply_masked<BPL>(mlist, mmask, mcnt, lane, x, y, z, soft2, ax, ay, az);
        __syncwarp();
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

template <int BPL, int WARPS>
static int launch_exact_shape(GroupedParams &P, cudaStream_t st) {
    const size_t smem = exact_smem<BPL>(WARPS);
    CNB_CUDA(cudaFuncSetAttribute(k_forces_exact<BPL, WARPS>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_forces_exact<BPL, WARPS>, WARPS * 32,
                                                  smem);
    // persistent grid: the work counter hands out buckets
    k_forces_exact<BPL, WARPS><<<kSMs * (per_sm > 0 ? per_sm : 1), WARPS * 32, smem, st>>>(P);
    return launch_status();
}

int launch_exact(GroupedParams &P, int bodies_per_lane, int block_warps, cudaStream_t st) {
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
