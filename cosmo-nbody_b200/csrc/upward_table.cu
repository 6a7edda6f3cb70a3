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

// Forms parent p from this node (s, lo, hi, moment qa/qb) and its sibling
// (bs, blo, bhi, ba/bb): tree_kernels.py:174-188 (left + right), min, max;
// writes the sums, the traversal record and (QUAD) the moment and b_max, and
// leaves the parent's values in s, lo, hi, qa, qb.
template <bool QUAD>
__device__ __forceinline__ void form_node(int64_t p, int2 ch, bool mine_left, float4 &s,
                                          float4 &lo, float4 &hi, float4 &qa, float4 &qb,
                                          float4 bs, float4 blo, float4 bhi, float4 ba,
                                          float4 bb, float4 *sums, float4 *rec, float4 *aabb,
                                          float4 *quad, bool keep_sums = true) {
    const float4 &Ls = mine_left ? s : bs, &Rs = mine_left ? bs : s;
    const float4 &Llo = mine_left ? lo : blo, &Rlo = mine_left ? blo : lo;
    const float4 &Lhi = mine_left ? hi : bhi, &Rhi = mine_left ? bhi : hi;
    const float4 qs = make_float4(__fadd_rn(Ls.x, Rs.x), __fadd_rn(Ls.y, Rs.y),
                                  __fadd_rn(Ls.z, Rs.z), __fadd_rn(Ls.w, Rs.w));
    const float4 qlo = make_float4(umin(Llo.x, Rlo.x), umin(Llo.y, Rlo.y), umin(Llo.z, Rlo.z), 0.f);
    const float4 qhi = make_float4(umax(Lhi.x, Rhi.x), umax(Lhi.y, Rhi.y), umax(Lhi.z, Rhi.z), 0.f);
    if (keep_sums) sums[p] = qs;  // the raw sums are read again only by climbs
    store_record(rec, aabb, p, qs, qlo, qhi, ch.x, ch.y);
    if (QUAD) {
        // left child first, then right: the same bits whichever child arrives second
        const float4 &La = mine_left ? qa : ba, &Ra = mine_left ? ba : qa;
        const float4 &Lb = mine_left ? qb : bb, &Rb = mine_left ? bb : qb;
        const float3 cp = centre_of(qs), cl = centre_of(Ls), cr = centre_of(Rs);
        float4 na = make_float4(__fadd_rn(La.x, Ra.x), __fadd_rn(La.y, Ra.y), __fadd_rn(La.z, Ra.z),
                                __fadd_rn(La.w, Ra.w));
        float4 nb = make_float4(__fadd_rn(Lb.x, Rb.x), __fadd_rn(Lb.y, Rb.y), 0.f, 0.f);
        moment_add(na, nb, Ls.w, __fsub_rn(cl.x, cp.x), __fsub_rn(cl.y, cp.y), __fsub_rn(cl.z, cp.z));
        moment_add(na, nb, Rs.w, __fsub_rn(cr.x, cp.x), __fsub_rn(cr.y, cp.y), __fsub_rn(cr.z, cp.z));
        quad[2 * p] = na;
        quad[2 * p + 1] = nb;
        const float bx = fmaxf(__fsub_rn(cp.x, qlo.x), __fsub_rn(qhi.x, cp.x));
        const float by = fmaxf(__fsub_rn(cp.y, qlo.y), __fsub_rn(qhi.y, cp.y));
        const float bz = fmaxf(__fsub_rn(cp.z, qlo.z), __fsub_rn(qhi.z, cp.z));
        rec[2 * p + 1].y = __fsqrt_rn(__fmaf_rn(bx, bx, __fmaf_rn(by, by, __fmul_rn(bz, bz))));
        qa = na;
        qb = nb;
    }
    s = qs;
    lo = qlo;
    hi = qhi;
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
        if (p == -1) break;
        if (p < 0 || p >= m_nodes) {
            set_flag(status, CNB_FLAG_BAD_TOPOLOGY);
            break;
        }
        // the topology of this level and the next is read while the
        // counter's atomic is in flight (it does not depend on it)
        const int2 ch = __ldg(children + p);
        const int32_t pp = __ldg(parents + p);
        // release this node's data, acquire the sibling's: the first arrival stops
        if (atomic_add_acq_rel(counts + p, 1) == 0) break;
        const bool mine_left = (ch.x == curr);
        const int32_t sib = mine_left ? ch.y : ch.x;
        if ((!mine_left && ch.y != curr) || sib == curr || sib < 0 || sib >= m_nodes) {
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
// The same pass in two phases over the bucket table (maximal subtrees of at
// most kUpSlots bodies): one warp per bucket forms every node inside its
// bucket with shared-memory counters and keeps the nodes' data in shared
// memory, so a level costs a shared-memory atomic instead of an L2 round
// trip; then one thread per bucket root climbs the levels above with the
// global counters.  Every node is still formed as (left + right) of its
// children: the table is bit-identical to the one-phase pass.
constexpr int kUpSlots = 64;  // leaves of a bucket; its internal nodes use as many slots
constexpr int kUpWarps = 4;

template <bool QUAD>
__global__ void __launch_bounds__(kUpWarps * 32) k_upward_buckets(
    const float *__restrict__ px, const float *__restrict__ py, const float *__restrict__ pz,
    const float *__restrict__ mass, const int2 *__restrict__ children,
    const int32_t *__restrict__ parents, const int32_t *__restrict__ ws, float4 *sums,
    float4 *rec, float4 *aabb, float4 *quad, int64_t n, int32_t *status) {
    // slot k < kUpSlots: leaf lo + k; slot kUpSlots + k: internal node n + lo + k
    __shared__ float4 s_sum[kUpWarps][2 * kUpSlots], s_lo[kUpWarps][2 * kUpSlots],
        s_hi[kUpWarps][2 * kUpSlots];
    __shared__ float4 s_qa[QUAD ? kUpWarps : 1][QUAD ? 2 * kUpSlots : 1],
        s_qb[QUAD ? kUpWarps : 1][QUAD ? 2 * kUpSlots : 1];
    __shared__ int s_cnt[kUpWarps][kUpSlots];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int nb = ws[0];
    const int4 *buckets = reinterpret_cast<const int4 *>(ws + 4);
    for (int g = blockIdx.x * kUpWarps + w; g < nb; g += gridDim.x * kUpWarps) {
        const int4 bk = buckets[g];
        const int lo_b = bk.x, count = bk.y;
        const int64_t root = bk.z;
        if (count < 1 || count > kUpSlots) {
            if (lane == 0) set_flag(status, CNB_FLAG_LIST_OVERFLOW);
            continue;
        }
        for (int k = lane; k < kUpSlots; k += 32) s_cnt[w][k] = 0;
        __syncwarp();
        for (int k = lane; k < count; k += 32) {
            const int64_t i = lo_b + k;
            const float m = mass[i], x = px[i], y = py[i], z = pz[i];
            float4 s = make_float4(__fmul_rn(x, m), __fmul_rn(y, m), __fmul_rn(z, m), m);
            float4 lo = make_float4(x, y, z, 0.f), hi = lo;
            float4 qa = make_float4(0.f, 0.f, 0.f, 0.f), qb = qa;
            // raw sums go to global memory only for the bucket root (phase two reads them)
            if (i == root) sums[i] = s;
            store_record(rec, aabb, i, s, lo, hi, -1, -1);
            s_sum[w][k] = s;
            s_lo[w][k] = lo;
            s_hi[w][k] = hi;
            if (QUAD) {
                s_qa[w][k] = qa;
                s_qb[w][k] = qb;
            }
            int64_t curr = i;
            for (int guard = 0; curr != root; ++guard) {
                const int32_t p = parents[curr];
                const int64_t ps = (int64_t)p - n - lo_b;
                if (guard > 2 * kUpSlots || ps < 0 || ps >= count) {
                    set_flag(status, CNB_FLAG_BAD_TOPOLOGY);
                    break;
                }
                const int2 ch = __ldg(children + p);
                __threadfence_block();  // this node's data before the count
                if (atomicAdd(&s_cnt[w][ps], 1) == 0) break;
                __threadfence_block();  // the sibling's data after the count
                const bool mine_left = (ch.x == curr);
                const int32_t sib = mine_left ? ch.y : ch.x;
                const int64_t so = sib < n ? (int64_t)sib - lo_b : kUpSlots + (int64_t)sib - n - lo_b;
                const int64_t lim = sib < n ? count : kUpSlots + count;
                if ((!mine_left && ch.y != curr) || sib == curr || sib < 0 ||
                    so < (sib < n ? 0 : kUpSlots) || so >= lim) {
                    set_flag(status, CNB_FLAG_BAD_TOPOLOGY);
                    break;
                }
                const float4 bs = s_sum[w][so], blo = s_lo[w][so], bhi = s_hi[w][so];
                float4 ba = make_float4(0.f, 0.f, 0.f, 0.f), bb = ba;
                if (QUAD) {
                    ba = s_qa[w][so];
                    bb = s_qb[w][so];
                }
                form_node<QUAD>(p, ch, mine_left, s, lo, hi, qa, qb, bs, blo, bhi, ba, bb, sums, rec,
                                aabb, quad, p == root);
                const int ns = kUpSlots + (int)ps;
                s_sum[w][ns] = s;
                s_lo[w][ns] = lo;
                s_hi[w][ns] = hi;
                if (QUAD) {
                    s_qa[w][ns] = qa;
                    s_qb[w][ns] = qb;
                }
                curr = p;
            }
        }
        __syncwarp();
    }
}

// Phase two: from every bucket root to the tree's root.
template <bool QUAD>
__global__ void __launch_bounds__(128) k_upward_roots(
    const int2 *__restrict__ children, const int32_t *__restrict__ parents,
    const int32_t *__restrict__ ws, int32_t *counts, float4 *sums, float4 *rec, float4 *aabb,
    float4 *quad, int64_t n, int32_t *status) {
    const int nb = ws[0];
    const int4 *buckets = reinterpret_cast<const int4 *>(ws + 4);
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < nb; g += gridDim.x * blockDim.x) {
        const int64_t root = buckets[g].z;
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
    if (quad)
        k_upward_buckets<true><<<kSMs * 8, kUpWarps * 32, 0, st>>>(
            px, py, pz, mass, ch, parents, workspace, s4, rec, rec + 2 * m, q4, n, status);
    else
        k_upward_buckets<false><<<kSMs * 8, kUpWarps * 32, 0, st>>>(
            px, py, pz, mass, ch, parents, workspace, s4, rec, rec + 2 * m, nullptr, n, status);
    CNB_TRY(launch_status());
    if (quad)
        k_upward_roots<true><<<kSMs * 4, 128, 0, st>>>(ch, parents, workspace, counts, s4, rec,
                                                       rec + 2 * m, q4, n, status);
    else
        k_upward_roots<false><<<kSMs * 4, 128, 0, st>>>(ch, parents, workspace, counts, s4, rec,
                                                        rec + 2 * m, nullptr, n, status);
    return launch_status();
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
