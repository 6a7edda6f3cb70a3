// tree.cu -- Karras radix-tree build and the upward (multipole) pass
// (src/kernels/tree_kernels.py:17-313).
//
// Layout: M = 2N-1 nodes, leaves 0..N-1 (sorted bodies), internal node of
// split i is N+i, root N.  children [M,2] int32 (-1 for leaves), parents [M]
// (-1 for the root), n_mass [M], n_com/n_min/n_max [M,3] float32.
#include "common.cuh"

namespace cnb {

// ---------------------------------------------------------------- reset
__global__ void k_reset_tree(int32_t *__restrict__ child, int32_t *__restrict__ parent,
                             int32_t *__restrict__ counters, int32_t *__restrict__ root_idx,
                             int64_t m) {
    int64_t i0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i0 == 0 && root_idx) root_idx[0] = 0;
    for (int64_t i = i0; i < m; i += (int64_t)gridDim.x * blockDim.x) {
        child[2 * i] = -1;
        child[2 * i + 1] = -1;
        parent[i] = -1;
        counters[i] = 0;
    }
}

// ---------------------------------------------------------------- build
// tree_kernels.py:36-58 delta_fn; equal keys -> 64 + (63 - clz64(i ^ j)).
__device__ __forceinline__ int delta_fn(const uint64_t *__restrict__ codes, uint64_t ki,
                                        int64_t i, int64_t j, int64_t n) {
    if (j < 0 || j >= n) return -1;
    uint64_t kj = __ldg(codes + j);
    if (ki == kj) return 64 + (63 - __clzll((long long)(i ^ j)));
    return __clzll((long long)(ki ^ kj));
}

// delta_fn with 32-bit indices (n <= 2^29, so i + 2 n stays below 2^31):
// the same values; for i != j, 63 - clz64(i ^ j) = 31 - clz32(i ^ j), and
// i == j gives 63 in both forms.
__device__ __forceinline__ int delta_fn32(const uint64_t *__restrict__ codes, uint64_t ki, int i,
                                          int j, int n) {
    if ((unsigned)j >= (unsigned)n) return -1;
    const uint64_t kj = __ldg(codes + j);
    if (ki == kj) return 64 + (31 - __clz(i ^ j));
    return __clzll((long long)(ki ^ kj));
}

// tree_kernels.py:60-129: the range [lo, hi] of split i's node, its split
// position gamma and its two children.  I: int64_t, or int for n <= 2^29
// (the same search, half the instructions).
struct Split {
    int64_t lo, hi, gamma;
    int32_t c0, c1;
};

template <typename I>
__device__ __forceinline__ int delta_any(const uint64_t *__restrict__ codes, uint64_t ki, I i, I j,
                                         I n) {
    if constexpr (sizeof(I) == 4) return delta_fn32(codes, ki, i, j, n);
    else return delta_fn(codes, ki, i, j, n);
}

template <typename I>
__device__ __forceinline__ Split split_of(const uint64_t *__restrict__ codes, I i, I n) {
    const uint64_t ki = __ldg(codes + i);
    const int d_prev = delta_any<I>(codes, ki, i, i - 1, n);
    const int d_next = delta_any<I>(codes, ki, i, i + 1, n);
    const I dir = d_next > d_prev ? 1 : -1;
    const int min_delta = d_next > d_prev ? d_prev : d_next;
    I l_max = 2;
    while (delta_any<I>(codes, ki, i, i + l_max * dir, n) > min_delta) l_max *= 2;
    I l = 0;
    for (I t = l_max >> 1; t >= 1; t >>= 1)  // t > 0: the reference's t // 2
        if (delta_any<I>(codes, ki, i, i + (l + t) * dir, n) > min_delta) l += t;
    const I j = i + l * dir;
    const int delta_node = delta_any<I>(codes, ki, i, j, n);
    I s = 0;
    for (I t = l; t > 0;) {
        I step = (t + 1) >> 1;
        if (delta_any<I>(codes, ki, i, i + (s + step) * dir, n) > delta_node) s += step;
        t -= step;
    }
    Split r;
    I gamma = i + s * dir;
    if (dir == -1) gamma -= 1;
    r.gamma = gamma;
    r.lo = i < j ? i : j;
    r.hi = i < j ? j : i;
    r.c0 = (int32_t)(r.lo == r.gamma ? r.gamma : r.gamma + n);
    r.c1 = (int32_t)(r.hi == r.gamma + 1 ? r.gamma + 1 : r.gamma + 1 + n);
    return r;
}

// tree_kernels.py:60-129 build_tree, one thread per split i < n-1.
__global__ void __launch_bounds__(256) k_build_tree(const uint64_t *__restrict__ codes,
                                                    int32_t *__restrict__ children,
                                                    int32_t *__restrict__ parents, int64_t n,
                                                    int2 *__restrict__ ranges) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n - 1;
         i += (int64_t)gridDim.x * blockDim.x) {
        const Split q = split_of<int64_t>(codes, i, n);
        const int64_t idx = i + n;
        children[2 * idx] = q.c0;
        children[2 * idx + 1] = q.c1;
        parents[q.c0] = (int32_t)idx;
        parents[q.c1] = (int32_t)idx;
        if (ranges) ranges[i] = make_int2((int)q.lo, (int)q.hi);
    }
}

// The bodies' (index + 1) summed over a bucket, modulo 2^32.  Summed over a
// bucket table it is n (n + 1) / 2 when the buckets tile the bodies once; a
// body in no bucket or in two moves it.  The bucketed upward pass checks it,
// and checks the topology inside every bucket: the reference's tie rule for
// equal keys (64 + 63 - clz(i ^ j), larger for farther indices) can build a
// tree in which some node has no parent and another has two.
__host__ __device__ __forceinline__ unsigned bucket_checksum(int64_t lo, int64_t size) {
    const uint64_t a = (uint64_t)lo + 1, b = (uint64_t)(lo + size);  // first and last index + 1
    return (unsigned)(((a + b) * (uint64_t)size) / 2);
}

// Bucket table for the grouped traversal: the maximal subtrees holding at
// most `max_size` bodies (a node qualifies when it is small enough and its
// parent is not).  Such buckets are contiguous in the sorted order and
// spatially compact (a radix-tree node covers one key prefix).  Appended in
// any order; ws[0] receives the count and ws[3] the table's checksum,
// ws[1] (the traversal's work counter) is reset.
__global__ void __launch_bounds__(256) k_make_buckets(const int2 *__restrict__ ranges,
                                                      const int32_t *__restrict__ parents,
                                                      int64_t n, int max_size,
                                                      int32_t *__restrict__ ws,
                                                      int4 *__restrict__ buckets,
                                                      const uint64_t *__restrict__ codes,
                                                      int box_shift) {
    const int64_t m = 2 * n - 1;
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < m;
         v += (int64_t)gridDim.x * blockDim.x) {
        int lo, size;
        if (v < n) {
            lo = (int)v;
            size = 1;
        } else {
            const int2 r = ranges[v - n];
            lo = r.x;
            size = r.y - r.x + 1;
        }
        if (size > max_size) continue;
        // with several boxes in the tree a bucket never spans two boxes
        if (codes && (codes[lo] >> box_shift) != (codes[lo + size - 1] >> box_shift)) continue;
        const int32_t p = parents[v];
        bool top = (p < 0);
        if (!top) {
            const int2 pr = ranges[p - n];
            top = (pr.y - pr.x + 1) > max_size ||
                  (codes && (codes[pr.x] >> box_shift) != (codes[pr.y] >> box_shift));
        }
        if (top) {
            const int slot = atomicAdd(ws, 1);
            buckets[slot] = make_int4(lo, size, (int)v, 0);
            atomicAdd(reinterpret_cast<unsigned *>(ws + 3), bucket_checksum(lo, size));
        }
    }
}

// Appends this warp's buckets of one table: for every lane's node holding more
// than max_size bodies, each child holding at most max_size (e0: the left
// child [lo, gamma], e1: the right child [gamma + 1, hi]), and the root when
// the whole tree fits (er).  One atomic per warp; every lane of the warp calls.
__device__ __forceinline__ void append_buckets(int32_t *ws, bool e0, bool e1, bool er, int lo,
                                               int gamma, int hi, int32_t c0, int32_t c1,
                                               int32_t root) {
    const unsigned b0 = __ballot_sync(0xffffffffu, e0), b1 = __ballot_sync(0xffffffffu, e1),
                   br = __ballot_sync(0xffffffffu, er);
    const int n0 = __popc(b0), n1 = __popc(b1), total = n0 + n1 + __popc(br);
    if (total == 0) return;
    const int lane = threadIdx.x & 31;
    int base = 0;
    if (lane == 0) base = atomicAdd(ws, total);
    base = __shfl_sync(0xffffffffu, base, 0);
    const unsigned lt = (1u << lane) - 1u;
    int4 *buckets = reinterpret_cast<int4 *>(ws + 4);
    unsigned sum = 0;
    if (e0) {
        buckets[base + __popc(b0 & lt)] = make_int4(lo, gamma - lo + 1, c0, 0);
        sum += bucket_checksum(lo, gamma - lo + 1);
    }
    if (e1) {
        buckets[base + n0 + __popc(b1 & lt)] = make_int4(gamma + 1, hi - gamma, c1, 0);
        sum += bucket_checksum(gamma + 1, hi - gamma);
    }
    if (er) {
        buckets[base + n0 + n1 + __popc(br & lt)] = make_int4(lo, hi - lo + 1, root, 0);
        sum += bucket_checksum(lo, hi - lo + 1);
    }
    sum = __reduce_add_sync(0xffffffffu, sum);
    if (lane == 0) atomicAdd(reinterpret_cast<unsigned *>(ws + 3), sum);
}

// The build fused with the bookkeeping of a grouped step: one thread per
// split i forms internal node n + i exactly as k_build_tree does, records
// its body range, zeroes its climb counter and appends its bucket children
// to the bucket table (ws, buckets of at most max_size bodies) and, when
// sws is given, to the super-bucket table (at most super_size): the same
// sets k_make_buckets finds, in another order.  The root is always node n
// (no split has node n as a child), so root_idx is written here and the
// root's parent, like the leaves' children, keeps the -1 it was given
// before the first build.  The loop is warp-uniform for the ballots.
template <typename I>
__global__ void __launch_bounds__(256) k_build_tree_buckets(
    const uint64_t *__restrict__ codes, int32_t *__restrict__ children,
    int32_t *__restrict__ parents, int64_t n, int2 *__restrict__ ranges,
    int32_t *__restrict__ counters, int32_t *__restrict__ root_idx, int max_size,
    int32_t *__restrict__ ws, int super_size, int32_t *__restrict__ sws) {
    const int lane = threadIdx.x & 31;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t base = blockIdx.x * (int64_t)blockDim.x + (threadIdx.x & ~31); base < n - 1;
         base += stride) {
        const int64_t i = base + lane;
        const bool valid = i < n - 1;
        int64_t lo = 0, hi = 0, gamma = 0;
        int32_t c0 = -1, c1 = -1;
        if (valid) {
            const Split q = split_of<I>(codes, (I)i, (I)n);
            lo = q.lo;
            hi = q.hi;
            gamma = q.gamma;
            c0 = q.c0;
            c1 = q.c1;
            const int64_t idx = i + n;
            reinterpret_cast<int2 *>(children)[idx] = make_int2(c0, c1);
            parents[c0] = (int32_t)idx;
            parents[c1] = (int32_t)idx;
            ranges[i] = make_int2((int)lo, (int)hi);
            counters[idx] = 0;
            if (i == 0 && root_idx) root_idx[0] = (int32_t)n;
        }
        const int64_t size = hi - lo + 1, s0 = gamma - lo + 1, s1 = hi - gamma;
        const int32_t root = (int32_t)n;
        append_buckets(ws, valid && size > max_size && s0 <= max_size,
                       valid && size > max_size && s1 <= max_size,
                       valid && i == 0 && size <= max_size, (int)lo, (int)gamma, (int)hi, c0, c1,
                       root);
        if (sws)
            append_buckets(sws, valid && size > super_size && s0 <= super_size,
                           valid && size > super_size && s1 <= super_size,
                           valid && i == 0 && size <= super_size, (int)lo, (int)gamma, (int)hi, c0,
                           c1, root);
    }
}

// ---------------------------------------------------------------- upward
// Numba's min/max of two floats (numba/cpython/builtins.py do_minmax).
__device__ __forceinline__ float pmin(float a, float b) { return b < a ? b : a; }
__device__ __forceinline__ float pmax(float a, float b) { return b > a ? b : a; }

struct Acc {
    float m, cx, cy, cz;      // mass and mass-weighted position sums
    float em, ex, ey, ez;     // compensation terms (compensated mode)
    float lx, ly, lz, hx, hy, hz;
};

// Exact error of a + b (Knuth two-sum; additions only, immune to FMA contraction).
__device__ __forceinline__ float two_sum_err(float a, float b, float s) {
    float bb = __fsub_rn(s, a);
    return __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
}

// tree_kernels.py:131-191 compute_multipoles.  One thread per leaf; the
// second arrival at a node (atomic counter) forms it from its two children
// as (left + right) and climbs on.  The counter increment is an acq_rel
// atomic: it releases the node's data and acquires the sibling's, which are
// then read through L2.  No thread ever waits.  A climb longer
// than the node count flags CNB_FLAG_BAD_TOPOLOGY and stops.
template <bool COMP>
__global__ void __launch_bounds__(256) k_upward(const float *__restrict__ px,
                                                const float *__restrict__ py,
                                                const float *__restrict__ pz,
                                                const float *__restrict__ mass,
                                                const int32_t *__restrict__ children,
                                                const int32_t *__restrict__ parents,
                                                float *n_mass, float *n_com, float *n_min,
                                                float *n_max, float *n_err, int32_t *counts,
                                                int64_t n, int32_t *status) {
    const int64_t m_nodes = 2 * n - 1;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        Acc a;
        a.m = mass[i];
        float x = px[i], y = py[i], z = pz[i];
        a.cx = __fmul_rn(x, a.m);
        a.cy = __fmul_rn(y, a.m);
        a.cz = __fmul_rn(z, a.m);
        a.lx = a.hx = x;
        a.ly = a.hy = y;
        a.lz = a.hz = z;
        n_mass[i] = a.m;
        n_com[3 * i] = a.cx;
        n_com[3 * i + 1] = a.cy;
        n_com[3 * i + 2] = a.cz;
        n_min[3 * i] = x;
        n_min[3 * i + 1] = y;
        n_min[3 * i + 2] = z;
        n_max[3 * i] = x;
        n_max[3 * i + 1] = y;
        n_max[3 * i + 2] = z;
        if (COMP) {
            a.em = 0.f;
            a.ex = __fmaf_rn(x, a.m, -a.cx);  // exact product error
            a.ey = __fmaf_rn(y, a.m, -a.cy);
            a.ez = __fmaf_rn(z, a.m, -a.cz);
            reinterpret_cast<float4 *>(n_err)[i] = make_float4(a.em, a.ex, a.ey, a.ez);
        }
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
            // this level's and the next level's topology are read while the
            // counter's atomic is in flight (they do not depend on it)
            const int32_t l = __ldg(children + 2 * p), r = __ldg(children + 2 * p + 1);
            const int32_t pp = __ldg(parents + p);
            // release this node's data, acquire the sibling's: the first arrival stops
            if (atomic_add_acq_rel(counts + p, 1) == 0) break;
            const bool mine_left = (l == curr);
            const int32_t s = mine_left ? r : l;
            if ((!mine_left && r != curr) || s == curr || s < 0 || s >= m_nodes) {
                set_flag(status, CNB_FLAG_BAD_TOPOLOGY);
                break;
            }
            Acc b;
            b.m = __ldcg(n_mass + s);
            b.cx = __ldcg(n_com + 3 * s);
            b.cy = __ldcg(n_com + 3 * s + 1);
            b.cz = __ldcg(n_com + 3 * s + 2);
            b.lx = __ldcg(n_min + 3 * s);
            b.ly = __ldcg(n_min + 3 * s + 1);
            b.lz = __ldcg(n_min + 3 * s + 2);
            b.hx = __ldcg(n_max + 3 * s);
            b.hy = __ldcg(n_max + 3 * s + 1);
            b.hz = __ldcg(n_max + 3 * s + 2);
            const Acc &L = mine_left ? a : b;
            const Acc &R = mine_left ? b : a;
            Acc q;
            q.m = __fadd_rn(L.m, R.m);
            q.cx = __fadd_rn(L.cx, R.cx);
            q.cy = __fadd_rn(L.cy, R.cy);
            q.cz = __fadd_rn(L.cz, R.cz);
            q.lx = pmin(L.lx, R.lx);
            q.ly = pmin(L.ly, R.ly);
            q.lz = pmin(L.lz, R.lz);
            q.hx = pmax(L.hx, R.hx);
            q.hy = pmax(L.hy, R.hy);
            q.hz = pmax(L.hz, R.hz);
            if (COMP) {
                float4 e = __ldcg(reinterpret_cast<const float4 *>(n_err) + s);
                b.em = e.x;
                b.ex = e.y;
                b.ey = e.z;
                b.ez = e.w;
                q.em = __fadd_rn(__fadd_rn(L.em, R.em), two_sum_err(L.m, R.m, q.m));
                q.ex = __fadd_rn(__fadd_rn(L.ex, R.ex), two_sum_err(L.cx, R.cx, q.cx));
                q.ey = __fadd_rn(__fadd_rn(L.ey, R.ey), two_sum_err(L.cy, R.cy, q.cy));
                q.ez = __fadd_rn(__fadd_rn(L.ez, R.ez), two_sum_err(L.cz, R.cz, q.cz));
                reinterpret_cast<float4 *>(n_err)[p] = make_float4(q.em, q.ex, q.ey, q.ez);
            }
            n_mass[p] = q.m;
            n_com[3 * p] = q.cx;
            n_com[3 * p + 1] = q.cy;
            n_com[3 * p + 2] = q.cz;
            n_min[3 * p] = q.lx;
            n_min[3 * p + 1] = q.ly;
            n_min[3 * p + 2] = q.lz;
            n_max[3 * p] = q.hx;
            n_max[3 * p + 1] = q.hy;
            n_max[3 * p + 2] = q.hz;
            a = q;
            curr = p;
            p = pp;
        }
    }
}

// tree_kernels.py:193-214 normalize_com: inv = 1.0 / m in float64, com * inv
// in float64, stored as float32.
__global__ void __launch_bounds__(256) k_normalize(const float *__restrict__ n_mass,
                                                   float *__restrict__ n_com, int64_t m) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m;
         i += (int64_t)gridDim.x * blockDim.x) {
        float mi = n_mass[i];
        if (mi > 0.f) {
            double inv = __ddiv_rn(1.0, (double)mi);
            n_com[3 * i] = __double2float_rn(__dmul_rn((double)n_com[3 * i], inv));
            n_com[3 * i + 1] = __double2float_rn(__dmul_rn((double)n_com[3 * i + 1], inv));
            n_com[3 * i + 2] = __double2float_rn(__dmul_rn((double)n_com[3 * i + 2], inv));
        }
    }
}

// Compensated normalisation: mass = m + em, com = (c + ec) / (m + em), float64.
__global__ void __launch_bounds__(256) k_normalize_comp(float *__restrict__ n_mass,
                                                        float *__restrict__ n_com,
                                                        const float4 *__restrict__ n_err,
                                                        int64_t m) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m;
         i += (int64_t)gridDim.x * blockDim.x) {
        float4 e = n_err[i];
        double mt = (double)n_mass[i] + (double)e.x;
        if (mt > 0.0) {
            double inv = 1.0 / mt;
            n_com[3 * i] = (float)(((double)n_com[3 * i] + (double)e.y) * inv);
            n_com[3 * i + 1] = (float)(((double)n_com[3 * i + 1] + (double)e.z) * inv);
            n_com[3 * i + 2] = (float)(((double)n_com[3 * i + 2] + (double)e.w) * inv);
        }
        n_mass[i] = (float)mt;
    }
}

// Float64 root reduction: sum m and m*x over all bodies (grid-stride, warp
// shuffles, one atomicAdd per warp into acc[4]).
__global__ void __launch_bounds__(256) k_root_f64(const float *__restrict__ px,
                                                  const float *__restrict__ py,
                                                  const float *__restrict__ pz,
                                                  const float *__restrict__ mass, int64_t n,
                                                  double *__restrict__ acc) {
    double s[4] = {0, 0, 0, 0};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        double m = mass[i];
        s[0] += m;
        s[1] += m * (double)px[i];
        s[2] += m * (double)py[i];
        s[3] += m * (double)pz[i];
    }
#pragma unroll
    for (int k = 0; k < 4; ++k)
        for (int o = 16; o > 0; o >>= 1) s[k] += __shfl_xor_sync(0xffffffffu, s[k], o);
    if ((threadIdx.x & 31) == 0)
        for (int k = 0; k < 4; ++k) atomicAdd(acc + k, s[k]);
}

__global__ void k_root_store(const double *__restrict__ acc, float *n_mass, float *n_com,
                             int64_t root, double *root_out) {
    double m = acc[0];
    double inv = m > 0 ? 1.0 / m : 0.0;
    double c[3] = {acc[1] * inv, acc[2] * inv, acc[3] * inv};
    if (n_mass) {
        n_mass[root] = (float)m;
        for (int k = 0; k < 3; ++k) n_com[3 * root + k] = (float)c[k];
    }
    root_out[0] = m;
    for (int k = 0; k < 3; ++k) root_out[1 + k] = c[k];
}

// tree_kernels.py:216-234 find_root.
__global__ void k_find_root(const int32_t *__restrict__ parents, int32_t *root_idx, int64_t m) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m;
         i += (int64_t)gridDim.x * blockDim.x)
        if (parents[i] == -1) atomicExch(root_idx, (int32_t)i);
}

// tree_kernels.py:264-313 build_top_tree_cache: breadth-first list of the
// first cache_size nodes (one thread, as in the reference; <= 256 steps).
__global__ void k_top_cache(const int32_t *__restrict__ child, const int32_t *__restrict__ root_idx,
                            int32_t *top, int32_t *n2c, int32_t cache) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    int32_t root = root_idx[0];
    if (root == -1) return;
    top[0] = root;
    n2c[root] = 0;
    int32_t rd = 0, wr = 1;
    while (rd < wr && wr < cache) {
        int32_t curr = top[rd];
        int32_t c1 = child[2 * curr];
        if (c1 != -1 && wr < cache) {
            top[wr] = c1;
            n2c[c1] = wr;
            wr++;
        }
        int32_t c2 = child[2 * curr + 1];
        if (c2 != -1 && wr < cache) {
            top[wr] = c2;
            n2c[c2] = wr;
            wr++;
        }
        rd++;
    }
    while (wr < cache) top[wr++] = -1;
}

}  // namespace cnb

using namespace cnb;

extern "C" int cnb_reset_tree_buffers(int32_t *child, int32_t *parent, int32_t *counters,
                                      int32_t *root_idx, int64_t n_nodes, void *stream) {
    if (n_nodes < 0 || (n_nodes > 0 && (!child || !parent || !counters))) return CNB_E_INVALID_ARG;
    if (n_nodes == 0 && !root_idx) return CNB_OK;
    k_reset_tree<<<grid_for(n_nodes > 0 ? n_nodes : 1, 256), 256, 0, as_stream(stream)>>>(
        child, parent, counters, root_idx, n_nodes);
    return launch_status();
}

extern "C" int cnb_build_tree(const uint64_t *codes, int32_t *children, int32_t *parents,
                              int64_t n, void *stream) {
    if (n < 0 || (n > 1 && (!codes || !children || !parents))) return CNB_E_INVALID_ARG;
    if (2 * n - 1 > (int64_t)INT32_MAX) return CNB_E_TOO_LARGE;
    if (n < 2) return CNB_OK;
    k_build_tree<<<grid_for(n - 1, 256), 256, 0, as_stream(stream)>>>(codes, children, parents,
                                                                       n, nullptr);
    return launch_status();
}

extern "C" int cnb_build_tree_ranges(const uint64_t *codes, int32_t *children, int32_t *parents,
                                     int32_t *ranges, int64_t n, void *stream) {
    if (n < 0 || (n > 1 && (!codes || !children || !parents || !ranges))) return CNB_E_INVALID_ARG;
    if ((reinterpret_cast<uintptr_t>(ranges) & 7) != 0) return CNB_E_INVALID_ARG;
    if (2 * n - 1 > (int64_t)INT32_MAX) return CNB_E_TOO_LARGE;
    if (n < 2) return CNB_OK;
    k_build_tree<<<grid_for(n - 1, 256), 256, 0, as_stream(stream)>>>(
        codes, children, parents, n, reinterpret_cast<int2 *>(ranges));
    return launch_status();
}

static int make_buckets(const int32_t *ranges, const int32_t *parents, const uint64_t *codes,
                        int box_shift, int64_t n, int max_size, int32_t *workspace,
                        void *stream) {
    if (n < 0 || max_size < 1 || !workspace) return CNB_E_INVALID_ARG;
    if (n > 1 && (!ranges || !parents)) return CNB_E_INVALID_ARG;
    if ((reinterpret_cast<uintptr_t>(workspace) & 15) != 0) return CNB_E_INVALID_ARG;
    cudaStream_t st = as_stream(stream);
    CNB_CUDA(cudaMemsetAsync(workspace, 0, 16, st));
    int4 *buckets = reinterpret_cast<int4 *>(workspace + 4);
    if (n == 0) return CNB_OK;
    if (n == 1) {
        const int32_t one[4] = {1, 0, 0, 1};  // one bucket; checksum 1
        const int32_t b[4] = {0, 1, 0, 0};
        CNB_CUDA(cudaMemcpyAsync(workspace, one, sizeof(one), cudaMemcpyHostToDevice, st));
        CNB_CUDA(cudaMemcpyAsync(buckets, b, sizeof(b), cudaMemcpyHostToDevice, st));
        return CNB_OK;
    }
    k_make_buckets<<<grid_for(2 * n - 1, 256), 256, 0, st>>>(
        reinterpret_cast<const int2 *>(ranges), parents, n, max_size, workspace, buckets, codes,
        box_shift);
    return launch_status();
}

extern "C" int cnb_make_buckets(const int32_t *ranges, const int32_t *parents, int64_t n,
                                int max_size, int32_t *workspace, void *stream) {
    return make_buckets(ranges, parents, nullptr, 0, n, max_size, workspace, stream);
}

extern "C" int cnb_make_buckets_boxes(const int32_t *ranges, const int32_t *parents,
                                      const uint64_t *codes, int box_bits, int64_t n,
                                      int max_size, int32_t *workspace, void *stream) {
    if (!codes || box_bits < 0 || box_bits > 30) return CNB_E_INVALID_ARG;
    return make_buckets(ranges, parents, codes, 3 * ((63 - box_bits) / 3), n, max_size,
                        workspace, stream);
}

extern "C" int cnb_build_tree_buckets(const uint64_t *codes, int32_t *children, int32_t *parents,
                                      int32_t *ranges, int32_t *counters, int32_t *root_idx,
                                      int64_t n, int max_size, int32_t *workspace, int super_size,
                                      int32_t *super_ws, void *stream) {
    if (n < 0 || max_size < 1 || !workspace || !root_idx) return CNB_E_INVALID_ARG;
    if (super_ws && super_size < 1) return CNB_E_INVALID_ARG;
    if (n > 1 && (!codes || !children || !parents || !ranges || !counters)) return CNB_E_INVALID_ARG;
    if ((reinterpret_cast<uintptr_t>(ranges) & 7) || (reinterpret_cast<uintptr_t>(children) & 7) ||
        (reinterpret_cast<uintptr_t>(workspace) & 15) || (reinterpret_cast<uintptr_t>(super_ws) & 15))
        return CNB_E_INVALID_ARG;
    if (2 * n - 1 > (int64_t)INT32_MAX) return CNB_E_TOO_LARGE;
    cudaStream_t st = as_stream(stream);
    if (n < 2) {
        // one body (or none): the root is leaf 0 and the only bucket
        CNB_CUDA(cudaMemsetAsync(root_idx, 0, 4, st));
        CNB_TRY(make_buckets(ranges, parents, nullptr, 0, n, max_size, workspace, stream));
        if (super_ws) CNB_TRY(make_buckets(ranges, parents, nullptr, 0, n, super_size, super_ws, stream));
        return CNB_OK;
    }
    CNB_CUDA(cudaMemsetAsync(workspace, 0, 16, st));
    if (super_ws) CNB_CUDA(cudaMemsetAsync(super_ws, 0, 16, st));
    if (n <= (int64_t)1 << 29)
        k_build_tree_buckets<int><<<grid_for(n - 1, 256), 256, 0, st>>>(
            codes, children, parents, n, reinterpret_cast<int2 *>(ranges), counters, root_idx,
            max_size, workspace, super_ws ? super_size : 0, super_ws);
    else
        k_build_tree_buckets<int64_t><<<grid_for(n - 1, 256), 256, 0, st>>>(
            codes, children, parents, n, reinterpret_cast<int2 *>(ranges), counters, root_idx,
            max_size, workspace, super_ws ? super_size : 0, super_ws);
    return launch_status();
}

static int upward_impl(const float *px, const float *py, const float *pz, const float *mass,
                       const int32_t *children, const int32_t *parents, float *n_mass,
                       float *n_com, float *n_min, float *n_max, float *n_err, int32_t *counts,
                       int64_t n, bool comp, int32_t *status, cudaStream_t st) {
    if (comp)
        k_upward<true><<<grid_for(n, 256), 256, 0, st>>>(px, py, pz, mass, children, parents,
                                                         n_mass, n_com, n_min, n_max, n_err,
                                                         counts, n, status);
    else
        k_upward<false><<<grid_for(n, 256), 256, 0, st>>>(px, py, pz, mass, children, parents,
                                                          n_mass, n_com, n_min, n_max, nullptr,
                                                          counts, n, status);
    return launch_status();
}

extern "C" int cnb_compute_multipoles(const float *px, const float *py, const float *pz,
                                      const float *mass, const int32_t *children,
                                      const int32_t *parents, float *n_mass, float *n_com,
                                      float *n_min, float *n_max, int32_t *counts, int64_t n,
                                      int32_t *status, void *stream) {
    if (n < 0) return CNB_E_INVALID_ARG;
    if (n == 0) return CNB_OK;
    if (!px || !py || !pz || !mass || !children || !parents || !n_mass || !n_com || !n_min ||
        !n_max || !counts)
        return CNB_E_INVALID_ARG;
    if (2 * n - 1 > (int64_t)INT32_MAX) return CNB_E_TOO_LARGE;
    return upward_impl(px, py, pz, mass, children, parents, n_mass, n_com, n_min, n_max, nullptr,
                       counts, n, false, status, as_stream(stream));
}

extern "C" int cnb_normalize_com(const float *n_mass, float *n_com, int64_t n_nodes,
                                 void *stream) {
    if (n_nodes < 0 || (n_nodes > 0 && (!n_mass || !n_com))) return CNB_E_INVALID_ARG;
    if (n_nodes == 0) return CNB_OK;
    k_normalize<<<grid_for(n_nodes, 256), 256, 0, as_stream(stream)>>>(n_mass, n_com, n_nodes);
    return launch_status();
}

extern "C" int cnb_upward(const float *px, const float *py, const float *pz, const float *mass,
                          const int32_t *children, const int32_t *parents, float *n_mass,
                          float *n_com, float *n_min, float *n_max, float *n_err,
                          int32_t *counts, int64_t n, int mode, double *root_f64,
                          int32_t *status, void *stream) {
    if (n < 0 || (mode != CNB_UPWARD_PLAIN && mode != CNB_UPWARD_COMPENSATED))
        return CNB_E_INVALID_ARG;
    if (n == 0) return CNB_OK;
    if (!px || !py || !pz || !mass || !children || !parents || !n_mass || !n_com || !n_min ||
        !n_max || !counts)
        return CNB_E_INVALID_ARG;
    const bool comp = (mode == CNB_UPWARD_COMPENSATED);
    if (comp && (!n_err || (reinterpret_cast<uintptr_t>(n_err) & 15))) return CNB_E_INVALID_ARG;
    if (comp && !root_f64) return CNB_E_INVALID_ARG;
    if (2 * n - 1 > (int64_t)INT32_MAX) return CNB_E_TOO_LARGE;
    cudaStream_t st = as_stream(stream);
    const int64_t m = 2 * n - 1;
    CNB_TRY(upward_impl(px, py, pz, mass, children, parents, n_mass, n_com, n_min, n_max, n_err,
                        counts, n, comp, status, st));
    const int64_t root = n > 1 ? n : 0;
    if (!comp) {
        k_normalize<<<grid_for(m, 256), 256, 0, st>>>(n_mass, n_com, m);
        CNB_TRY(launch_status());
        if (root_f64) {  // report the float64 root; the float32 tree stays bit-exact
            CNB_CUDA(cudaMemsetAsync(root_f64, 0, 4 * sizeof(double), st));
            k_root_f64<<<grid_for(n, 256, 148 * 4), 256, 0, st>>>(px, py, pz, mass, n, root_f64);
            CNB_TRY(launch_status());
            k_root_store<<<1, 1, 0, st>>>(root_f64, nullptr, nullptr, root, root_f64);
            CNB_TRY(launch_status());
        }
        return CNB_OK;
    }
    k_normalize_comp<<<grid_for(m, 256), 256, 0, st>>>(n_mass, n_com,
                                                       reinterpret_cast<const float4 *>(n_err), m);
    CNB_TRY(launch_status());
    CNB_CUDA(cudaMemsetAsync(root_f64, 0, 4 * sizeof(double), st));
    k_root_f64<<<grid_for(n, 256, 148 * 4), 256, 0, st>>>(px, py, pz, mass, n, root_f64);
    CNB_TRY(launch_status());
    k_root_store<<<1, 1, 0, st>>>(root_f64, n_mass, n_com, root, root_f64);
    return launch_status();
}

extern "C" int cnb_find_root(const int32_t *parents, int32_t *root_idx, int64_t n_nodes,
                             void *stream) {
    if (n_nodes < 0 || !root_idx || (n_nodes > 0 && !parents)) return CNB_E_INVALID_ARG;
    if (n_nodes == 0) return CNB_OK;
    k_find_root<<<grid_for(n_nodes, 256), 256, 0, as_stream(stream)>>>(parents, root_idx, n_nodes);
    return launch_status();
}

extern "C" int cnb_build_top_tree_cache(const int32_t *child, const int32_t *root_idx,
                                        int32_t *top_nodes, int32_t *node_to_cache,
                                        int32_t cache_size, void *stream) {
    if (!child || !root_idx || !top_nodes || !node_to_cache || cache_size < 1)
        return CNB_E_INVALID_ARG;
    k_top_cache<<<1, 1, 0, as_stream(stream)>>>(child, root_idx, top_nodes, node_to_cache,
                                                 cache_size);
    return launch_status();
}

