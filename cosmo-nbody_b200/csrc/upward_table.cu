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
__device__ __forceinline__ void moment_add(float4 &a, float4 &b, float m, float dx, float dy,
                                           float dz) {
    a.x = fmaf(m * dx, dx, a.x);
    a.y = fmaf(m * dx, dy, a.y);
    a.z = fmaf(m * dx, dz, a.z);
    a.w = fmaf(m * dy, dy, a.w);
    b.x = fmaf(m * dy, dz, b.x);
    b.y = fmaf(m * dz, dz, b.y);
}

__device__ __forceinline__ float3 centre_of(float4 s) {
    const float inv = s.w > 0.f ? 1.f / s.w : 0.f;
    return make_float3(s.x * inv, s.y * inv, s.z * inv);
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
    const int64_t m_nodes = 2 * n - 1;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const float m = mass[i], x = px[i], y = py[i], z = pz[i];
        // tree_kernels.py:152-159 leaf: com = p * m (float32), box = p
        float4 s = make_float4(__fmul_rn(x, m), __fmul_rn(y, m), __fmul_rn(z, m), m);
        float4 lo = make_float4(x, y, z, 0.f), hi = lo;
        float4 qa = make_float4(0.f, 0.f, 0.f, 0.f), qb = qa;  // this node's moment (QUAD)
        sums[i] = s;
        store_record(rec, aabb, i, s, lo, hi, -1, -1);
        int64_t curr = i;
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
            const float4 &Ls = mine_left ? s : bs, &Rs = mine_left ? bs : s;
            const float4 &Llo = mine_left ? lo : blo, &Rlo = mine_left ? blo : lo;
            const float4 &Lhi = mine_left ? hi : bhi, &Rhi = mine_left ? bhi : hi;
            // tree_kernels.py:174-188: (left + right), min, max
            const float4 qs = make_float4(__fadd_rn(Ls.x, Rs.x), __fadd_rn(Ls.y, Rs.y),
                                          __fadd_rn(Ls.z, Rs.z), __fadd_rn(Ls.w, Rs.w));
            const float4 qlo = make_float4(umin(Llo.x, Rlo.x), umin(Llo.y, Rlo.y),
                                           umin(Llo.z, Rlo.z), 0.f);
            const float4 qhi = make_float4(umax(Lhi.x, Rhi.x), umax(Lhi.y, Rhi.y),
                                           umax(Lhi.z, Rhi.z), 0.f);
            sums[p] = qs;
            store_record(rec, aabb, p, qs, qlo, qhi, ch.x, ch.y);
            if (QUAD) {
                float4 ba = make_float4(0.f, 0.f, 0.f, 0.f), bb = ba;
                if (sib >= n) {
                    ba = __ldcg(quad + 2 * sib);
                    bb = __ldcg(quad + 2 * sib + 1);
                }
                const float3 cp = centre_of(qs), cm = centre_of(s), cs = centre_of(bs);
                float4 na = make_float4(qa.x + ba.x, qa.y + ba.y, qa.z + ba.z, qa.w + ba.w);
                float4 nb = make_float4(qb.x + bb.x, qb.y + bb.y, 0.f, 0.f);
                moment_add(na, nb, s.w, cm.x - cp.x, cm.y - cp.y, cm.z - cp.z);
                moment_add(na, nb, bs.w, cs.x - cp.x, cs.y - cp.y, cs.z - cp.z);
                quad[2 * p] = na;
                quad[2 * p + 1] = nb;
                const float bx = fmaxf(cp.x - qlo.x, qhi.x - cp.x);
                const float by = fmaxf(cp.y - qlo.y, qhi.y - cp.y);
                const float bz = fmaxf(cp.z - qlo.z, qhi.z - cp.z);
                rec[2 * p + 1].y = sqrtf(fmaf(bx, bx, fmaf(by, by, bz * bz)));
                qa = na;
                qb = nb;
            }
            s = qs;
            lo = qlo;
            hi = qhi;
            curr = p;
            p = pp;
        }
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
