// upward_table.cu -- the upward pass of tree_kernels.py:131-214 written for
// the grouped traversal: one kernel forms every node's sums and box and
// writes its traversal record directly (normalised CoM, mass, extents,
// children), so no separate normalisation or packing pass runs.
//
// The climb keeps its working data packed: the raw mass-weighted sums of a
// node in one float4 (`sums`, scratch) and its box in the table's two boxes
// float4s, so a climb step reads its sibling with three 128-bit loads and
// writes the parent with five 128-bit stores.  The arithmetic is the
// reference's: float32 (left + right) sums, Numba min/max, CoM normalised as
// c * (1.0 / m) in float64 -- the table is bit-identical to the one built by
// cnb_upward + cnb_pack_nodes.  cnb_unpack_nodes writes the reference-layout
// arrays from the table when they are wanted.
#include "common.cuh"

namespace cnb {

__device__ __forceinline__ float umin(float a, float b) { return b < a ? b : a; }  // Numba min
__device__ __forceinline__ float umax(float a, float b) { return b > a ? b : a; }  // Numba max

__device__ __forceinline__ float4 normalised(float4 s) {
    if (s.w > 0.f) {  // tree_kernels.py:207-214: one reciprocal in float64
        const double inv = __ddiv_rn(1.0, (double)s.w);
        s.x = __double2float_rn(__dmul_rn((double)s.x, inv));
        s.y = __double2float_rn(__dmul_rn((double)s.y, inv));
        s.z = __double2float_rn(__dmul_rn((double)s.z, inv));
    }
    return s;
}

__device__ __forceinline__ void store_record(float4 *rec, float4 *aabb, int64_t v, float4 s,
                                             float4 lo, float4 hi, int32_t c0, int32_t c1) {
    const float sx = hi.x - lo.x;
    rec[2 * v] = normalised(s);
    rec[2 * v + 1] = make_float4(sx, fmaxf(sx, fmaxf(hi.y - lo.y, hi.z - lo.z)),
                                 __int_as_float(c0), __int_as_float(c1));
    aabb[2 * v] = lo;
    aabb[2 * v + 1] = hi;
}

// Second central moment of the union of two children (parallel-axis rule):
// M2 = M2_l + m_l (c_l - c)(c_l - c)^T + M2_r + m_r (c_r - c)(c_r - c)^T,
// six components (xx, xy, xz, yy, yz, zz) in two float4s.
// Explicit-rounding intrinsics throughout, so no compiler contraction makes
// the moments depend on which kernel forms a node.
__device__ __forceinline__ void moment_add(float4 &a, float4 &b, float m, float dx, float dy,
                                           float dz) {
    const float mx = __fmul_rn(m, dx), my = __fmul_rn(m, dy), mz = __fmul_rn(m, dz);
    a.x = __fmaf_rn(mx, dx, a.x);
    a.y = __fmaf_rn(mx, dy, a.y);
    a.z = __fmaf_rn(mx, dz, a.z);
    a.w = __fmaf_rn(my, dy, a.w);
    b.x = __fmaf_rn(my, dz, b.x);
    b.y = __fmaf_rn(mz, dz, b.y);
}

__device__ __forceinline__ float3 centre_of(float4 s) {
    const float inv = s.w > 0.f ? __frcp_rn(s.w) : 0.f;
    return make_float3(__fmul_rn(s.x, inv), __fmul_rn(s.y, inv), __fmul_rn(s.z, inv));
}

// The parent of children L and R: tree_kernels.py:174-188 (left + right),
// min, max, and (QUAD) the second central moment from the children's
// moments and centres, left child first, then right.
template <bool QUAD>
__device__ __forceinline__ void combine(float4 Ls, float4 Llo, float4 Lhi, float4 La, float4 Lb,
                                        float4 Rs, float4 Rlo, float4 Rhi, float4 Ra, float4 Rb,
                                        float4 &qs, float4 &qlo, float4 &qhi, float4 &na,
                                        float4 &nb) {
    qs = make_float4(__fadd_rn(Ls.x, Rs.x), __fadd_rn(Ls.y, Rs.y), __fadd_rn(Ls.z, Rs.z),
                     __fadd_rn(Ls.w, Rs.w));
    qlo = make_float4(umin(Llo.x, Rlo.x), umin(Llo.y, Rlo.y), umin(Llo.z, Rlo.z), 0.f);
    qhi = make_float4(umax(Lhi.x, Rhi.x), umax(Lhi.y, Rhi.y), umax(Lhi.z, Rhi.z), 0.f);
    if (QUAD) {
        const float3 cp = centre_of(qs), cl = centre_of(Ls), cr = centre_of(Rs);
        na = make_float4(__fadd_rn(La.x, Ra.x), __fadd_rn(La.y, Ra.y), __fadd_rn(La.z, Ra.z),
                         __fadd_rn(La.w, Ra.w));
        nb = make_float4(__fadd_rn(Lb.x, Rb.x), __fadd_rn(Lb.y, Rb.y), 0.f, 0.f);
        moment_add(na, nb, Ls.w, __fsub_rn(cl.x, cp.x), __fsub_rn(cl.y, cp.y), __fsub_rn(cl.z, cp.z));
        moment_add(na, nb, Rs.w, __fsub_rn(cr.x, cp.x), __fsub_rn(cr.y, cp.y), __fsub_rn(cr.z, cp.z));
    }
}

// Writes internal node p: its traversal record and box, its raw sums when
// keep_sums (read again only by climbs) and (QUAD) its moment, with b_max in
// the record's 3-D-extent slot.
template <bool QUAD>
__device__ __forceinline__ void write_node(int64_t p, float4 qs, float4 qlo, float4 qhi,
                                           float4 na, float4 nb, int2 ch, float4 *sums,
                                           float4 *rec, float4 *aabb, float4 *quad,
                                           bool keep_sums) {
    if (keep_sums) sums[p] = qs;
    const float sx = qhi.x - qlo.x;
    float ext = fmaxf(sx, fmaxf(qhi.y - qlo.y, qhi.z - qlo.z));
    if (QUAD) {
        quad[2 * p] = na;
        quad[2 * p + 1] = nb;
        const float3 cp = centre_of(qs);
        const float bx = fmaxf(__fsub_rn(cp.x, qlo.x), __fsub_rn(qhi.x, cp.x));
        const float by = fmaxf(__fsub_rn(cp.y, qlo.y), __fsub_rn(qhi.y, cp.y));
        const float bz = fmaxf(__fsub_rn(cp.z, qlo.z), __fsub_rn(qhi.z, cp.z));
        ext = __fsqrt_rn(__fmaf_rn(bx, bx, __fmaf_rn(by, by, __fmul_rn(bz, bz))));
    }
    rec[2 * p] = normalised(qs);
    rec[2 * p + 1] = make_float4(sx, ext, __int_as_float(ch.x), __int_as_float(ch.y));
    aabb[2 * p] = qlo;
    aabb[2 * p + 1] = qhi;
}

// Forms parent p from this node (s, lo, hi, moment qa/qb) and its sibling
// (bs, blo, bhi, ba/bb), writes it, and leaves the parent's values in s, lo,
// hi, qa, qb.
template <bool QUAD>
__device__ __forceinline__ void form_node(int64_t p, int2 ch, bool mine_left, float4 &s,
                                          float4 &lo, float4 &hi, float4 &qa, float4 &qb,
                                          float4 bs, float4 blo, float4 bhi, float4 ba,
                                          float4 bb, float4 *sums, float4 *rec, float4 *aabb,
                                          float4 *quad, bool keep_sums = true) {
    float4 qs, qlo, qhi, na = qa, nb = qb;
    if (mine_left)
        combine<QUAD>(s, lo, hi, qa, qb, bs, blo, bhi, ba, bb, qs, qlo, qhi, na, nb);
    else
        combine<QUAD>(bs, blo, bhi, ba, bb, s, lo, hi, qa, qb, qs, qlo, qhi, na, nb);
    write_node<QUAD>(p, qs, qlo, qhi, na, nb, ch, sums, rec, aabb, quad, keep_sums);
    s = qs;
    lo = qlo;
    hi = qhi;
    qa = na;
    qb = nb;
}

// One node's climb towards the root with the global atomic counters: the
// second arrival at a parent forms it as (left + right) and climbs on.
template <bool QUAD>
__device__ __forceinline__ void climb(int64_t curr, float4 s, float4 lo, float4 hi, float4 qa,
                                      float4 qb, const int2 *__restrict__ children,
                                      const int32_t *__restrict__ parents, int32_t *counts,
                                      float4 *sums, float4 *rec, float4 *aabb, float4 *quad,
                                      int64_t n, int32_t *status) {
    const int64_t m_nodes = 2 * n - 1;
    int32_t p = parents[curr];
    for (int64_t guard = 0;; ++guard) {
        if (guard > m_nodes) {
            set_flag(status, CNB_FLAG_BAD_TOPOLOGY);
            break;
        }
        if (p == -1) {
            // only the tree's root (node n; leaf 0 for one body) has no parent
            if (curr != (n > 1 ? n : 0)) set_flag(status, CNB_FLAG_BAD_TOPOLOGY);
            break;
        }
        if (p < 0 || p >= m_nodes) {
            set_flag(status, CNB_FLAG_BAD_TOPOLOGY);
            break;
        }
        // the topology of this level and the next is read while the
        // counter's atomic is in flight (it does not depend on it)
        const int2 ch = __ldg(children + p);
        const int32_t pp = __ldg(parents + p);
        // release this node's data, acquire the sibling's: the first arrival stops
        // (after the check that p is this node's parent, which every arrival makes)
        const int32_t arrived = atomic_add_acq_rel(counts + p, 1);
        const bool mine_left = (ch.x == curr);
        if (!mine_left && ch.y != curr) {
            set_flag(status, CNB_FLAG_BAD_TOPOLOGY);
            break;
        }
        if (arrived == 0) break;
        const int32_t sib = mine_left ? ch.y : ch.x;
        if (sib == curr || sib < 0 || sib >= m_nodes) {
            set_flag(status, CNB_FLAG_BAD_TOPOLOGY);
            break;
        }
        const float4 bs = __ldcg(sums + sib);
        const float4 blo = __ldcg(aabb + 2 * sib), bhi = __ldcg(aabb + 2 * sib + 1);
        float4 ba = make_float4(0.f, 0.f, 0.f, 0.f), bb = ba;
        if (QUAD && sib >= n) {
            ba = __ldcg(quad + 2 * sib);
            bb = __ldcg(quad + 2 * sib + 1);
        }
        form_node<QUAD>(p, ch, mine_left, s, lo, hi, qa, qb, bs, blo, bhi, ba, bb, sums, rec, aabb,
                        quad);
        curr = p;
        p = pp;
    }
}

// QUAD: also the second central moment of every internal node, quad[2v],
// quad[2v + 1] (leaves hold none: a leaf's moment is zero and is never read),
// and in the record's 3-D-extent slot the node's b_max instead: the largest
// distance from its CoM to a corner of its box (no member lies farther), the
// size the periodic-law opening test needs once quadrupoles are applied.
template <bool QUAD>
__global__ void __launch_bounds__(256) k_upward_table(
    const float *__restrict__ px, const float *__restrict__ py, const float *__restrict__ pz,
    const float *__restrict__ mass, const int2 *__restrict__ children,
    const int32_t *__restrict__ parents, int32_t *counts, float4 *sums, float4 *rec, float4 *aabb,
    float4 *quad, int64_t n, int32_t *status) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const float m = mass[i], x = px[i], y = py[i], z = pz[i];
        // tree_kernels.py:152-159 leaf: com = p * m (float32), box = p
        const float4 s = make_float4(__fmul_rn(x, m), __fmul_rn(y, m), __fmul_rn(z, m), m);
        const float4 lo = make_float4(x, y, z, 0.f);
        const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
        sums[i] = s;
        store_record(rec, aabb, i, s, lo, lo, -1, -1);
        climb<QUAD>(i, s, lo, lo, zero, zero, children, parents, counts, sums, rec, aabb, quad, n,
                    status);
    }
}

// ---------------------------------------------------------------- by buckets
// The same pass over the bucket table (maximal subtrees of at most kUpSlots
// bodies), one warp per bucket, level by level in shared memory.  A
// radix-tree subtree over bodies [lo, hi] whose root is node n + lo holds the
// internal nodes n + lo .. n + hi - 1, one whose root is n + hi holds
// n + lo + 1 .. n + hi (the left child of a node is named by its last body,
// the right child by its first), so the bucket's children are one coalesced
// read.  The warp checks that they form a tree over the bucket's bodies
// (every body and node but the root has exactly one parent), loads the
// leaves, and then forms, round after round, every node whose two children
// are ready; each lane owns at most two of the bucket's nodes, no lane waits
// on another and no atomic is needed; the records are written afterwards,
// consecutive nodes on consecutive lanes.  Every node is formed as
// (left + right) of its children: the table is bit-identical to the
// one-phase pass.  After every 32 buckets a warp climbs on above their
// roots, one lane each, with the global counters (the first arrival at a
// node stops, as in the one-phase pass).
constexpr int kUpSlots = 64;  // leaves of a bucket; its internal nodes use as many slots
constexpr int kUpWarps = 4;

// Climbs above the bucket roots one lane each (root < 0: nothing), reading a
// root's sums and box back from global memory; the roots were formed by
// other lanes of this warp, whose writes the fence and the warp barrier
// order before this lane's release at the first counter.
template <bool QUAD>
__device__ __forceinline__ void climb_roots(int64_t root, const int2 *__restrict__ children,
                                            const int32_t *__restrict__ parents, int32_t *counts,
                                            float4 *sums, float4 *rec, float4 *aabb, float4 *quad,
                                            int64_t n, int32_t *status) {
    __threadfence();
    __syncwarp();
    if (root >= 0) {
        const float4 s = __ldcg(sums + root);
        const float4 lo = __ldcg(aabb + 2 * root), hi = __ldcg(aabb + 2 * root + 1);
        float4 qa = make_float4(0.f, 0.f, 0.f, 0.f), qb = qa;
        if (QUAD && root >= n) {
            qa = __ldcg(quad + 2 * root);
            qb = __ldcg(quad + 2 * root + 1);
        }
        climb<QUAD>(root, s, lo, hi, qa, qb, children, parents, counts, sums, rec, aabb, quad, n,
                    status);
    }
    __syncwarp();
}

template <bool QUAD>
__global__ void __launch_bounds__(kUpWarps * 32) k_upward_buckets(
    const float *__restrict__ px, const float *__restrict__ py, const float *__restrict__ pz,
    const float *__restrict__ mass, const int2 *__restrict__ children,
    const int32_t *__restrict__ parents, const int32_t *__restrict__ ws, int32_t *counts,
    float4 *sums, float4 *rec, float4 *aabb, float4 *quad, int64_t n, int32_t *status) {
    // slot k < kUpSlots: leaf lo + k; slot kUpSlots + k: internal node n + lo + k
    __shared__ float4 s_sum[kUpWarps][2 * kUpSlots], s_lo[kUpWarps][2 * kUpSlots],
        s_hi[kUpWarps][2 * kUpSlots];
    __shared__ float4 s_qa[QUAD ? kUpWarps : 1][QUAD ? 2 * kUpSlots : 1],
        s_qb[QUAD ? kUpWarps : 1][QUAD ? 2 * kUpSlots : 1];
    __shared__ int s_par[kUpWarps][2 * kUpSlots];  // parent (internal index) of each slot
    __shared__ int s_rdy[kUpWarps][2 * kUpSlots];  // the slot's data is in shared memory
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int nb = ws[0];
    const int4 *buckets = reinterpret_cast<const int4 *>(ws + 4);
    // the buckets tile the bodies once (the table's checksum, see bucket_checksum)
    if (blockIdx.x == 0 && threadIdx.x == 0 &&
        (unsigned)ws[3] != (unsigned)((uint64_t)n * (uint64_t)(n + 1) / 2))
        set_flag(status, CNB_FLAG_BAD_TOPOLOGY);
    int64_t my_root = -1;  // the bucket root this lane climbs from
    const int stride = gridDim.x * kUpWarps;
    int4 bk_next = make_int4(0, 0, 0, 0);
    if (blockIdx.x * kUpWarps + w < nb) bk_next = buckets[blockIdx.x * kUpWarps + w];
    for (int g = blockIdx.x * kUpWarps + w, t = 0; g < nb; g += stride, ++t) {
        if (t > 0 && (t & 31) == 0) {
            climb_roots<QUAD>(my_root, children, parents, counts, sums, rec, aabb, quad, n, status);
            my_root = -1;
        }
        const int4 bk = bk_next;
        if (g + stride < nb) bk_next = buckets[g + stride];  // in flight during this bucket
        const int lo_b = bk.x, count = bk.y;
        const int64_t root = bk.z;
        const int off = (count > 1 && root == n + lo_b + count - 1) ? 1 : 0;  // first internal slot
        const int root_slot = count == 1 ? 0 : kUpSlots + (int)(root - n - lo_b);
        if (count > kUpSlots) {
            if (lane == 0) set_flag(status, CNB_FLAG_LIST_OVERFLOW);
            continue;
        }
        if (count < 1 || lo_b < 0 || (int64_t)lo_b + count > n || root >= 2 * n - 1 ||
            (count == 1 ? root != lo_b : root != n + lo_b && root != n + lo_b + count - 1)) {
            if (lane == 0) set_flag(status, CNB_FLAG_BAD_TOPOLOGY);
            continue;
        }
        // every global read of the bucket at once: its leaves and its internal nodes' children
        float4 leaf[2];  // (x, y, z, m) of bodies lo + lane and lo + lane + 32
        int2 chn[2];
        bool own[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int k = lane + 32 * h;
            leaf[h] = make_float4(0.f, 0.f, 0.f, 0.f);
            if (k < count) {
                const int64_t i = lo_b + k;
                leaf[h] = make_float4(px[i], py[i], pz[i], mass[i]);
            }
            own[h] = off + k < off + count - 1;
            chn[h] = own[h] ? __ldg(children + n + lo_b + off + k) : make_int2(-1, -1);
        }
        for (int k = lane; k < 2 * kUpSlots; k += 32) {
            s_par[w][k] = -1;
            s_rdy[w][k] = k < count;  // the leaves are ready once stored
        }
        __syncwarp();
        // this lane's internal nodes: slots kUpSlots + off + lane (+ 32), children at a[][]
        int a[2][2];
        bool bad = false;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int k = off + lane + 32 * h;
            a[h][0] = a[h][1] = 0;
            if (!own[h]) continue;
            bool ok = true;
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                const int64_t v = c == 0 ? chn[h].x : chn[h].y;
                const int64_t r = v < n ? v - lo_b : v - n - lo_b;
                ok = ok && v >= 0 && (v < n ? r >= 0 && r < count : r >= off && r < off + count - 1);
                a[h][c] = ok ? (v < n ? (int)r : kUpSlots + (int)r) : 0;
            }
            if (ok && a[h][0] != a[h][1])
                bad |= (atomicExch(&s_par[w][a[h][0]], k) != -1) |
                       (atomicExch(&s_par[w][a[h][1]], k) != -1);
            else
                bad = true;
        }
        __syncwarp();
        // a tree: every slot but the root has exactly one parent, the root none
        for (int k = lane; k < count; k += 32) bad |= (s_par[w][k] < 0) != (k == root_slot);
        for (int k = off + lane; k < off + count - 1; k += 32)
            bad |= (s_par[w][kUpSlots + k] < 0) != (kUpSlots + k == root_slot);
        if (__any_sync(0xffffffffu, bad)) {
            if (lane == 0) set_flag(status, CNB_FLAG_BAD_TOPOLOGY);
            continue;
        }
        // the leaves
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int k = lane + 32 * h;
            if (k >= count) continue;
            const int64_t i = lo_b + k;
            const float x = leaf[h].x, y = leaf[h].y, z = leaf[h].z, m = leaf[h].w;
            const float4 sv = make_float4(__fmul_rn(x, m), __fmul_rn(y, m), __fmul_rn(z, m), m);
            const float4 lv = make_float4(x, y, z, 0.f);
            // raw sums go to global memory only for the bucket root (the climb above reads them)
            if (i == root) sums[i] = sv;
            store_record(rec, aabb, i, sv, lv, lv, -1, -1);
            s_sum[w][k] = sv;
            s_lo[w][k] = lv;
            s_hi[w][k] = lv;
            if (QUAD) s_qa[w][k] = s_qb[w][k] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
        __syncwarp();
        // the internal nodes, round by round (a round forms every node whose
        // children are ready; a valid bucket needs at most count - 1 rounds)
        bool done[2] = {!own[0], !own[1]};
        for (int round = 0; round < count; ++round) {
            bool formed[2] = {false, false};
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                if (done[h] || !s_rdy[w][a[h][0]] || !s_rdy[w][a[h][1]]) continue;
                const int l = a[h][0], r = a[h][1], ns = kUpSlots + off + lane + 32 * h;
                const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
                float4 qs, qlo, qhi, na = zero, nb = zero;
                combine<QUAD>(s_sum[w][l], s_lo[w][l], s_hi[w][l], QUAD ? s_qa[w][l] : zero,
                              QUAD ? s_qb[w][l] : zero, s_sum[w][r], s_lo[w][r], s_hi[w][r],
                              QUAD ? s_qa[w][r] : zero, QUAD ? s_qb[w][r] : zero, qs, qlo, qhi, na,
                              nb);
                s_sum[w][ns] = qs;
                s_lo[w][ns] = qlo;
                s_hi[w][ns] = qhi;
                if (QUAD) {
                    s_qa[w][ns] = na;
                    s_qb[w][ns] = nb;
                }
                formed[h] = true;
            }
            __syncwarp();  // the data of this round's nodes before their flags
#pragma unroll
            for (int h = 0; h < 2; ++h)
                if (formed[h]) {
                    s_rdy[w][kUpSlots + off + lane + 32 * h] = 1;
                    done[h] = true;
                }
            __syncwarp();
            if (!__any_sync(0xffffffffu, !(done[0] && done[1]))) break;
        }
        // a cycle among the internal nodes leaves some of them unformed
        if (__any_sync(0xffffffffu, !(done[0] && done[1]))) {
            if (lane == 0) set_flag(status, CNB_FLAG_BAD_TOPOLOGY);
            continue;
        }
        // the records of the bucket's internal nodes, consecutive nodes on consecutive lanes
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            if (!own[h]) continue;
            const int k = off + lane + 32 * h, ns = kUpSlots + k;
            const int64_t p = n + lo_b + k;
            write_node<QUAD>(p, s_sum[w][ns], s_lo[w][ns], s_hi[w][ns],
                             QUAD ? s_qa[w][ns] : make_float4(0.f, 0.f, 0.f, 0.f),
                             QUAD ? s_qb[w][ns] : make_float4(0.f, 0.f, 0.f, 0.f), chn[h], sums,
                             rec, aabb, quad, p == root);
        }
        if (lane == (t & 31)) my_root = root;
    }
    climb_roots<QUAD>(my_root, children, parents, counts, sums, rec, aabb, quad, n, status);
}

// Reference-layout node arrays from the traversal table (octree.py:85-93
// get_buffers): n_mass, normalised n_com, n_min, n_max.
__global__ void __launch_bounds__(256) k_unpack_nodes(const float4 *__restrict__ rec,
                                                      const float4 *__restrict__ aabb,
                                                      float *__restrict__ n_mass,
                                                      float *__restrict__ n_com,
                                                      float *__restrict__ n_min,
                                                      float *__restrict__ n_max, int64_t m) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < m;
         v += (int64_t)gridDim.x * blockDim.x) {
        const float4 a = rec[2 * v], lo = aabb[2 * v], hi = aabb[2 * v + 1];
        n_mass[v] = a.w;
        n_com[3 * v] = a.x;
        n_com[3 * v + 1] = a.y;
        n_com[3 * v + 2] = a.z;
        n_min[3 * v] = lo.x;
        n_min[3 * v + 1] = lo.y;
        n_min[3 * v + 2] = lo.z;
        n_max[3 * v] = hi.x;
        n_max[3 * v + 1] = hi.y;
        n_max[3 * v + 2] = hi.z;
    }
}

}  // namespace cnb

using namespace cnb;

extern "C" int cnb_upward_table(const float *px, const float *py, const float *pz,
                                const float *mass, const int32_t *children,
                                const int32_t *parents, int32_t *counts, float *node_table,
                                float *sums, int64_t n, int32_t *status, void *stream) {
    if (n < 0) return CNB_E_INVALID_ARG;
    if (n == 0) return CNB_OK;
    if (!px || !py || !pz || !mass || !children || !parents || !counts || !node_table || !sums)
        return CNB_E_INVALID_ARG;
    if ((reinterpret_cast<uintptr_t>(node_table) & 15) || (reinterpret_cast<uintptr_t>(sums) & 15) ||
        (reinterpret_cast<uintptr_t>(children) & 7))
        return CNB_E_INVALID_ARG;
    if (2 * n - 1 > (int64_t)INT32_MAX) return CNB_E_TOO_LARGE;
    const int64_t m = 2 * n - 1;
    float4 *rec = reinterpret_cast<float4 *>(node_table);
    k_upward_table<false><<<grid_for(n, 256), 256, 0, as_stream(stream)>>>(
        px, py, pz, mass, reinterpret_cast<const int2 *>(children), parents, counts,
        reinterpret_cast<float4 *>(sums), rec, rec + 2 * m, nullptr, n, status);
    return launch_status();
}

extern "C" int cnb_upward_table_quad(const float *px, const float *py, const float *pz,
                                     const float *mass, const int32_t *children,
                                     const int32_t *parents, int32_t *counts, float *node_table,
                                     float *sums, float *quad, int64_t n, int32_t *status,
                                     void *stream) {
    if (n < 0) return CNB_E_INVALID_ARG;
    if (n == 0) return CNB_OK;
    if (!px || !py || !pz || !mass || !children || !parents || !counts || !node_table || !sums ||
        !quad)
        return CNB_E_INVALID_ARG;
    if ((reinterpret_cast<uintptr_t>(node_table) & 15) || (reinterpret_cast<uintptr_t>(sums) & 15) ||
        (reinterpret_cast<uintptr_t>(quad) & 15) || (reinterpret_cast<uintptr_t>(children) & 7))
        return CNB_E_INVALID_ARG;
    if (2 * n - 1 > (int64_t)INT32_MAX) return CNB_E_TOO_LARGE;
    const int64_t m = 2 * n - 1;
    float4 *rec = reinterpret_cast<float4 *>(node_table);
    k_upward_table<true><<<grid_for(n, 256), 256, 0, as_stream(stream)>>>(
        px, py, pz, mass, reinterpret_cast<const int2 *>(children), parents, counts,
        reinterpret_cast<float4 *>(sums), rec, rec + 2 * m, reinterpret_cast<float4 *>(quad), n,
        status);
    return launch_status();
}

template <bool QUAD>
static int launch_upward_buckets(const float *px, const float *py, const float *pz,
                                 const float *mass, const int2 *ch, const int32_t *parents,
                                 const int32_t *workspace, int32_t *counts, float4 *sums,
                                 float4 *rec, float4 *aabb, float4 *quad, int64_t n,
                                 int32_t *status, cudaStream_t st) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_upward_buckets<QUAD>, kUpWarps * 32, 0);
    k_upward_buckets<QUAD><<<kSMs * (per_sm > 0 ? per_sm : 1), kUpWarps * 32, 0, st>>>(
        px, py, pz, mass, ch, parents, workspace, counts, sums, rec, aabb, quad, n, status);
    return launch_status();
}

extern "C" int cnb_upward_table_buckets(const float *px, const float *py, const float *pz,
                                        const float *mass, const int32_t *children,
                                        const int32_t *parents, const int32_t *workspace,
                                        int32_t *counts, float *node_table, float *sums,
                                        float *quad, int64_t n, int32_t *status, void *stream) {
    if (n < 0) return CNB_E_INVALID_ARG;
    if (n == 0) return CNB_OK;
    if (!px || !py || !pz || !mass || !children || !parents || !workspace || !counts ||
        !node_table || !sums)
        return CNB_E_INVALID_ARG;
    if ((reinterpret_cast<uintptr_t>(node_table) & 15) || (reinterpret_cast<uintptr_t>(sums) & 15) ||
        (reinterpret_cast<uintptr_t>(quad) & 15) || (reinterpret_cast<uintptr_t>(children) & 7) ||
        (reinterpret_cast<uintptr_t>(workspace) & 15))
        return CNB_E_INVALID_ARG;
    if (2 * n - 1 > (int64_t)INT32_MAX) return CNB_E_TOO_LARGE;
    const int64_t m = 2 * n - 1;
    float4 *rec = reinterpret_cast<float4 *>(node_table);
    float4 *q4 = reinterpret_cast<float4 *>(quad);
    const int2 *ch = reinterpret_cast<const int2 *>(children);
    float4 *s4 = reinterpret_cast<float4 *>(sums);
    cudaStream_t st = as_stream(stream);
    // the bucket count is on the device: persistent grids over the buckets
    if (quad) return launch_upward_buckets<true>(px, py, pz, mass, ch, parents, workspace, counts,
                                                 s4, rec, rec + 2 * m, q4, n, status, st);
    return launch_upward_buckets<false>(px, py, pz, mass, ch, parents, workspace, counts, s4, rec,
                                        rec + 2 * m, nullptr, n, status, st);
}

extern "C" int cnb_unpack_nodes(const float *node_table, float *n_mass, float *n_com,
                                float *n_min, float *n_max, int64_t n_nodes, void *stream) {
    if (n_nodes < 0) return CNB_E_INVALID_ARG;
    if (n_nodes == 0) return CNB_OK;
    if (!node_table || !n_mass || !n_com || !n_min || !n_max) return CNB_E_INVALID_ARG;
    if (reinterpret_cast<uintptr_t>(node_table) & 15) return CNB_E_INVALID_ARG;
    const float4 *rec = reinterpret_cast<const float4 *>(node_table);
    k_unpack_nodes<<<grid_for(n_nodes, 256), 256, 0, as_stream(stream)>>>(
        rec, rec + 2 * n_nodes, n_mass, n_com, n_min, n_max, n_nodes);
    return launch_status();
}
