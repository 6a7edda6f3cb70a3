// forces_grouped.cu -- warp-cooperative Barnes-Hut traversal over
// Morton-contiguous leaf buckets (the B200 form of
// src/kernels/physics_kernels.py:14-153).
//
// One warp per bucket of 32 consecutive (Morton-sorted) bodies.  The warp
// walks the tree 32 nodes at a time from a per-warp node stack in shared
// memory: each lane tests one node against the bucket's bounding box, the
// accepted nodes (and reached leaves) are appended to a per-warp interaction
// list in shared memory with one ballot, and the opened nodes push their two
// children.  Whenever the list holds 32 entries every lane applies all of
// them to its own body (float32, rsqrt, per-pair minimum image), so the
// force loop reads shared memory only and runs without divergence.
//
// Opening tests (bucket box B, node CoM image c nearest the bucket centre,
// dmin = periodic distance from c to B, per axis):
//   CNB_MAC_REF_X:    open unless leaf or sx^2 < theta^2 dmin^2, sx the node's
//                     x-extent set to `box` above box/2 (physics_kernels.py:131-136).
//                     Every node the bucket accepts, each of its bodies would
//                     accept in the reference traversal (dmin <= |d|).
//   CNB_MAC_PERIODIC: 3-D extent l; also open any node whose image is not the
//                     same for every (body, node member) pair, so the monopole
//                     of an accepted node is applied at one consistent image.
// theta can be one value or one per bucket (learned controller).
#include "common.cuh"

namespace cnb {

constexpr int kGWarps = 4;           // warps per block
constexpr int kGStack = 2048;        // node stack entries per warp
constexpr int kGList = 64;           // interaction list entries per warp

struct GroupedParams {
    const float *px, *py, *pz;
    const float4 *nA;  // (com x, y, z, mass)
    const float4 *nB;  // (min x, y, z, child0 bits)
    const float4 *nC;  // (max x, y, z, child1 bits)
    float *force;      // [N,3]
    const float *theta_per_group;  // may be null
    float theta;
    float G, soft2, box;
    int mac;
    int64_t n;
    int64_t m_nodes;
    int32_t root;
    int64_t n_groups;
    unsigned long long *stats;  // [0] interactions, [1] node tests (may be null)
    int32_t *status;
};

__device__ __forceinline__ void apply_list(const float4 *list, int cnt, float x, float y,
                                           float z, float soft2, float &ax, float &ay,
                                           float &az) {
#pragma unroll 8
    for (int j = 0; j < cnt; ++j) {
        const float4 e = list[j];
        float dx = e.x - x, dy = e.y - y, dz = e.z - z;
        dx -= rintf(dx);
        dy -= rintf(dy);
        dz -= rintf(dz);
        const float d2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
        const float r = rsqrtf(d2 + soft2);
        const float f = (d2 > 1e-7f) ? e.w * r * r * r : 0.f;
        ax = fmaf(f, dx, ax);
        ay = fmaf(f, dy, ay);
        az = fmaf(f, dz, az);
    }
}

__global__ void __launch_bounds__(kGWarps * 32) k_forces_grouped(GroupedParams P) {
    __shared__ int32_t s_stack[kGWarps][kGStack];
    __shared__ float4 s_list[kGWarps][kGList];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const uint32_t lt = (1u << lane) - 1u;
    int32_t *stack = s_stack[wib];
    float4 *list = s_list[wib];
    unsigned long long n_inter = 0, n_tests = 0;
    bool overflow = false;

    for (int64_t g = (int64_t)blockIdx.x * kGWarps + wib; g < P.n_groups;
         g += (int64_t)gridDim.x * kGWarps) {
        const int64_t i = g * 32 + lane;
        const bool valid = i < P.n;
        const int64_t ii = valid ? i : g * 32;
        const float x = P.px[ii], y = P.py[ii], z = P.pz[ii];
        if (valid && !(isfinite(x) && isfinite(y) && isfinite(z))) set_flag(P.status, CNB_FLAG_NONFINITE);
        // bucket bounding box (Morton buckets are compact; the wrap-around
        // of a bucket across the periodic boundary is handled by the
        // per-axis periodic distance below only when the box is < box/2)
        float lx = x, ly = y, lz = z, hx = x, hy = y, hz = z;
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
        const float th = P.theta_per_group ? P.theta_per_group[g] : P.theta;
        const float th2 = th * th;
        const float half_box = 0.5f * P.box;

        float ax = 0.f, ay = 0.f, az = 0.f;
        int top = 0, cnt = 0;
        if (lane == 0) stack[0] = P.root;
        top = 1;
        __syncwarp();
        // a valid tree pushes every node at most once per bucket: more
        // rounds than nodes means a cyclic topology
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
            bool accept = false, open = false;
            float4 A;
            int32_t c0 = -1, c1 = -1;
            if (node >= P.m_nodes) {
                set_flag(P.status, CNB_FLAG_BAD_TOPOLOGY);
                node = -1;
            }
            if (node >= 0) {
                A = __ldg(P.nA + node);
                if (A.w > 0.f) {
                    const float4 B = __ldg(P.nB + node);
                    const float4 C = __ldg(P.nC + node);
                    c0 = __float_as_int(B.w);
                    c1 = __float_as_int(C.w);
                    if (c0 == -1) {
                        accept = true;
                    } else {
                        float dx = A.x - gcx, dy = A.y - gcy, dz = A.z - gcz;
                        const float sx_ = rintf(dx), sy_ = rintf(dy), sz_ = rintf(dz);
                        dx -= sx_;
                        dy -= sy_;
                        dz -= sz_;
                        const float tx = fmaxf(fabsf(dx) - ghx, 0.f);
                        const float ty = fmaxf(fabsf(dy) - ghy, 0.f);
                        const float tz = fmaxf(fabsf(dz) - ghz, 0.f);
                        const float d2min = tx * tx + ty * ty + tz * tz;
                        if (P.mac == CNB_MAC_REF_X) {
                            float s = C.x - B.x;
                            s = s > half_box ? P.box : s;
                            accept = s * s < th2 * d2min;
                        } else {
                            // node box at the image chosen for its CoM
                            const float ex = fmaxf(C.x - sx_, hx) - fminf(B.x - sx_, lx);
                            const float ey = fmaxf(C.y - sy_, hy) - fminf(B.y - sy_, ly);
                            const float ez = fmaxf(C.z - sz_, hz) - fminf(B.z - sz_, lz);
                            const bool consistent = ex < half_box && ey < half_box && ez < half_box;
                            const float l = fmaxf(C.x - B.x, fmaxf(C.y - B.y, C.z - B.z));
                            accept = consistent && (l * l < th2 * d2min);
                        }
                        open = !accept;
                    }
                }
            }
            n_tests += (node >= 0);
            const uint32_t am = __ballot_sync(0xffffffffu, accept);
            const uint32_t om = __ballot_sync(0xffffffffu, open);
            if (accept) list[cnt + __popc(am & lt)] = A;
            cnt += __popc(am);
            const int nopen = __popc(om);
            if (top + 2 * nopen > kGStack) {
                overflow = true;  // drop the children (flagged)
            } else {
                if (open) {
                    const int pos = top + 2 * __popc(om & lt);
                    stack[pos] = c1;
                    stack[pos + 1] = c0;
                }
                top += 2 * nopen;
            }
            __syncwarp();
            if (cnt >= 32) {
                apply_list(list, 32, x, y, z, P.soft2, ax, ay, az);
                n_inter += 32;
                __syncwarp();
                if (lane < cnt - 32) list[lane] = list[32 + lane];
                cnt -= 32;
                __syncwarp();
            }
        }
        apply_list(list, cnt, x, y, z, P.soft2, ax, ay, az);
        n_inter += cnt;
        __syncwarp();
        if (valid) {
            const float fx = P.G * ax, fy = P.G * ay, fz = P.G * az;
            P.force[3 * i] = fx;
            P.force[3 * i + 1] = fy;
            P.force[3 * i + 2] = fz;
            if (!isfinite(fx) || !isfinite(fy) || !isfinite(fz)) set_flag(P.status, CNB_FLAG_NONFINITE);
        }
    }
    if (overflow && lane == 0) set_flag(P.status, CNB_FLAG_LIST_OVERFLOW);
    if (P.stats && lane == 0) {
        // n_inter counts list entries per warp (each applied to 32 lanes)
        atomicAdd(P.stats, n_inter);
    }
    if (P.stats) {
        for (int o = 16; o > 0; o >>= 1) n_tests += __shfl_xor_sync(0xffffffffu, n_tests, o);
        if (lane == 0) atomicAdd(P.stats + 1, n_tests);
    }
}

// Node table for the grouped traversal from the reference-layout tree.
__global__ void __launch_bounds__(256) k_pack_nodes(const float *__restrict__ n_mass,
                                                    const float *__restrict__ n_com,
                                                    const float *__restrict__ n_min,
                                                    const float *__restrict__ n_max,
                                                    const int2 *__restrict__ children,
                                                    float4 *__restrict__ A, float4 *__restrict__ B,
                                                    float4 *__restrict__ C, int64_t m) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int2 ch = children[i];
        A[i] = make_float4(n_com[3 * i], n_com[3 * i + 1], n_com[3 * i + 2], n_mass[i]);
        B[i] = make_float4(n_min[3 * i], n_min[3 * i + 1], n_min[3 * i + 2], __int_as_float(ch.x));
        C[i] = make_float4(n_max[3 * i], n_max[3 * i + 1], n_max[3 * i + 2], __int_as_float(ch.y));
    }
}

}  // namespace cnb

using namespace cnb;

extern "C" int cnb_pack_nodes(const float *n_mass, const float *n_com, const float *n_min,
                              const float *n_max, const int32_t *children, float *node_table,
                              int64_t n_nodes, void *stream) {
    if (n_nodes < 0) return CNB_E_INVALID_ARG;
    if (n_nodes == 0) return CNB_OK;
    if (!n_mass || !n_com || !n_min || !n_max || !children || !node_table)
        return CNB_E_INVALID_ARG;
    if ((reinterpret_cast<uintptr_t>(node_table) & 15) || (reinterpret_cast<uintptr_t>(children) & 7))
        return CNB_E_INVALID_ARG;
    float4 *A = reinterpret_cast<float4 *>(node_table);
    k_pack_nodes<<<grid_for(n_nodes, 256), 256, 0, as_stream(stream)>>>(
        n_mass, n_com, n_min, n_max, reinterpret_cast<const int2 *>(children), A, A + n_nodes,
        A + 2 * n_nodes, n_nodes);
    return launch_status();
}

extern "C" int cnb_forces_grouped(const float *px, const float *py, const float *pz,
                                  const float *node_table, float *force, int64_t n, double theta,
                                  const float *theta_per_group, int mac, double G, double soft,
                                  double box, unsigned long long *stats, int32_t *status,
                                  void *stream) {
    if (n < 0 || (mac != CNB_MAC_REF_X && mac != CNB_MAC_PERIODIC)) return CNB_E_INVALID_ARG;
    if (n == 0) return CNB_OK;
    if (!px || !py || !pz || !node_table || !force) return CNB_E_INVALID_ARG;
    if (reinterpret_cast<uintptr_t>(node_table) & 15) return CNB_E_INVALID_ARG;
    if (2 * n - 1 > (int64_t)INT32_MAX) return CNB_E_TOO_LARGE;
    const int64_t m = 2 * n - 1;
    GroupedParams P;
    P.px = px;
    P.py = py;
    P.pz = pz;
    P.nA = reinterpret_cast<const float4 *>(node_table);
    P.nB = P.nA + m;
    P.nC = P.nA + 2 * m;
    P.force = force;
    P.theta_per_group = theta_per_group;
    P.theta = (float)theta;
    P.G = (float)G;
    P.soft2 = (float)(soft * soft);
    P.box = (float)box;
    P.mac = mac;
    P.n = n;
    P.m_nodes = m;
    P.root = n > 1 ? (int32_t)n : 0;
    P.n_groups = (n + 31) / 32;
    P.stats = stats;
    P.status = status;
    const int64_t blocks_needed = (P.n_groups + kGWarps - 1) / kGWarps;
    const int64_t cap = 148LL * 64;
    const int grid = (int)(blocks_needed < cap ? blocks_needed : cap);
    k_forces_grouped<<<grid, kGWarps * 32, 0, as_stream(stream)>>>(P);
    return launch_status();
}
