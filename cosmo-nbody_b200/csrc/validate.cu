// validate.cu -- topology check of a radix tree (no reference counterpart;
// the reference never checks its tree).  A valid tree over n bodies has
// n-1 internal nodes, every node except one root is the child of exactly
// one internal node, and parents[] agrees with children[].  Long runs of
// equal 30-bit keys can make the reference's tie rule build an invalid tree;
// this check turns that into CNB_FLAG_BAD_TOPOLOGY instead of wrong forces.
#include "common.cuh"

namespace cnb {

__global__ void __launch_bounds__(256) k_claims(const int2 *__restrict__ children,
                                                const int32_t *__restrict__ parents, int64_t n,
                                                int32_t *__restrict__ claims,
                                                int32_t *__restrict__ status) {
    const int64_t m = 2 * n - 1;
    for (int64_t p = n + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < m;
         p += (int64_t)gridDim.x * blockDim.x) {
        const int2 c = children[p];
        if (c.x < 0 || c.x >= m || c.y < 0 || c.y >= m || c.x == c.y) {
            set_flag(status, CNB_FLAG_BAD_TOPOLOGY);
            continue;
        }
        atomicAdd(claims + c.x, 1);
        atomicAdd(claims + c.y, 1);
        if (parents[c.x] != p || parents[c.y] != p) set_flag(status, CNB_FLAG_BAD_TOPOLOGY);
    }
}

__global__ void __launch_bounds__(256) k_check_claims(const int32_t *__restrict__ claims,
                                                      const int32_t *__restrict__ parents,
                                                      int64_t m, int32_t *__restrict__ roots,
                                                      int32_t *__restrict__ status) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < m;
         v += (int64_t)gridDim.x * blockDim.x) {
        const int32_t c = claims[v];
        if (parents[v] == -1) {
            atomicAdd(roots, 1);
            if (c != 0) set_flag(status, CNB_FLAG_BAD_TOPOLOGY);
        } else if (c != 1) {
            set_flag(status, CNB_FLAG_BAD_TOPOLOGY);
        }
    }
}

__global__ void k_check_roots(const int32_t *roots, int32_t *status) {
    if (*roots != 1) set_flag(status, CNB_FLAG_BAD_TOPOLOGY);
}

}  // namespace cnb

extern "C" int cnb_validate_tree(const int32_t *children, const int32_t *parents, int64_t n,
                                 int32_t *scratch, int32_t *status, void *stream) {
    if (n < 1 || !children || !parents || !scratch || !status) return CNB_E_INVALID_ARG;
    if ((reinterpret_cast<uintptr_t>(children) & 7) != 0) return CNB_E_INVALID_ARG;
    const int64_t m = 2 * n - 1;
    cudaStream_t st = cnb::as_stream(stream);
    CNB_CUDA(cudaMemsetAsync(scratch, 0, sizeof(int32_t) * (m + 1), st));
    if (n > 1) {
        cnb::k_claims<<<cnb::grid_for(n - 1, 256), 256, 0, st>>>(
            reinterpret_cast<const int2 *>(children), parents, n, scratch, status);
        CNB_TRY(cnb::launch_status());
    }
    cnb::k_check_claims<<<cnb::grid_for(m, 256), 256, 0, st>>>(scratch, parents, m, scratch + m,
                                                               status);
    CNB_TRY(cnb::launch_status());
    cnb::k_check_roots<<<1, 1, 0, st>>>(scratch + m, status);
    return cnb::launch_status();
}
