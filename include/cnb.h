/*
 * cnb.h -- C ABI of libcnb.so, the B200 (sm_100a) Barnes-Hut step.
 *
 * Each entry point replaces one Numba kernel (or CuPy call) of
 * Cosmo-NBody; the comment above it cites the reference interface it
 * stands in for.  Conventions:
 *   - all array arguments are device pointers owned by the caller, in the
 *     reference's layouts (SoA float32 positions/velocities, force [N,3]
 *     row-major, children [M,2] int32, n_com/n_min/n_max [M,3] float32,
 *     M = 2N-1 tree nodes: leaves 0..N-1, internal nodes N..2N-2);
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default);
 *   - every call is asynchronous on `stream` and returns 0 or a negative
 *     CNB_E_* code for argument or launch errors;
 *   - kernels that can detect a bad state on the device OR CNB_FLAG_* bits
 *     into `status` (one int32 in device memory, may be NULL); the caller
 *     reads it after synchronising;
 *   - no entry point allocates memory except cnb_ctx_create.
 */
#ifndef CNB_H
#define CNB_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* return codes */
#define CNB_OK 0
#define CNB_E_INVALID_ARG (-1)
#define CNB_E_CUDA (-2)
#define CNB_E_NO_MEMORY (-3)
#define CNB_E_TOO_LARGE (-4)
#define CNB_E_DEVICE_FLAG (-5)

/* device status bits */
#define CNB_FLAG_STACK_OVERFLOW 1 /* traversal stack full: children dropped (reference: silent) */
#define CNB_FLAG_BAD_TOPOLOGY 2   /* climb longer than the node count, or child index out of range */
#define CNB_FLAG_NONFINITE 4      /* non-finite acceleration produced */
#define CNB_FLAG_LIST_OVERFLOW 8  /* grouped traversal work queue exhausted */
#define CNB_FLAG_WAIT_LIMIT 16    /* a bounded wait between blocks gave up (result invalid) */
#define CNB_FLAG_SORT_CHECK 32    /* a destination check of the near-sorted path failed (result invalid) */

/* Morton key modes */
#define CNB_KEY_COMPAT30 0 /* bit-exact with morton.py:13-63 (low 10 bits of each 21-bit coordinate) */
#define CNB_KEY_MORTON63 1 /* full 21-bit interleave, coordinates clamped to [0, 2^21-1] */

/* opening criteria */
#define CNB_MAC_REF_X 0    /* physics_kernels.py:131-136: x-extent, clamped to box when > box/2,
                            decided per body (the grouped forms give every body the reference's
                            own node set) */
#define CNB_MAC_PERIODIC 1 /* 3-D extent, and open any node whose image is ambiguous for a target */
#define CNB_MAC_EWALD 2    /* periodic (Ewald) force law, 3-D extent: cnb_forces_grouped_ewald */
#define CNB_MAC_REF_X_BUCKET 3 /* the reference's test decided once per bucket against the bucket's
                                  box (a node opens unless every body of the bucket would accept
                                  it): finer node sets than the reference's, not its forces */

/* arithmetic of the per-particle traversal */
#define CNB_PREC_F32 0
#define CNB_PREC_F64 1 /* float64 like compiled Numba types physics_kernels.py:118-141 */

/* upward pass modes */
#define CNB_UPWARD_PLAIN 0       /* bit-exact with tree_kernels.py:131-214 */
#define CNB_UPWARD_COMPENSATED 1 /* two-sum compensated float32 sums, float64 root */

int cnb_version(void);
const char *cnb_error_string(int code);
/* Last CUDA error seen by the library on this host thread (cudaError_t value). */
int cnb_last_cuda_error(void);
/* Number of kernels this library has launched in this process. */
int64_t cnb_launch_count(void);

/* src/kernels/morton.py:65-90 compute_codes(pos_x, pos_y, pos_z, codes, indices, n_bodies).
 * indices may be NULL. */
int cnb_compute_codes(const float *x, const float *y, const float *z, uint64_t *codes,
                      uint32_t *indices, int64_t n, int key_mode, void *stream);

/* Scratch owner for the radix sort and the fused step. */
typedef struct cnb_ctx cnb_ctx;
int cnb_ctx_create(int64_t n_max, cnb_ctx **out);
int cnb_ctx_destroy(cnb_ctx *ctx);

/* src/core/state.py:35 `sort_idx = cp.argsort(codes)`: stable LSD radix
 * sort of (key, index) pairs.  keys_out receives the sorted keys, perm_out
 * the original index of each sorted key.  idx_in may be NULL (identity).
 * key_bits = number of low key bits that may be non-zero (30 or 63).
 * keys_out may be keys_in and perm_out may be idx_in (at least two passes
 * then run); any other overlap between the four arrays is rejected
 * (CNB_E_INVALID_ARG).
 * One kernel per 8-bit digit: each 4096-key tile finds where its keys go by
 * looking back at the counts earlier tiles publish; the waits are bounded,
 * and a wait that gives up raises CNB_FLAG_WAIT_LIMIT in the context
 * (cnb_ctx_take_flags). */
int cnb_sort_pairs(cnb_ctx *ctx, const uint64_t *keys_in, uint64_t *keys_out,
                   const uint32_t *idx_in, uint32_t *perm_out, int64_t n, int key_bits,
                   void *stream);

/* No counterpart in the reference.  Test hook for the sort's failure paths
 * (all off by default): wait_limit > 0 bounds every look-back wait of the
 * one-sweep sort at that many polls (0: the default 2^22); withheld_tile >= 0
 * makes that 4096-key tile of every pass keep its digit counts to itself, so
 * the tiles after it wait until their limit, give up and raise
 * CNB_FLAG_WAIT_LIMIT (-1: off); near_dest_bias > 0 shifts every destination
 * of the near-sorted path's placement by that many keys, so its destination
 * check skips the writes that leave the array and raises
 * CNB_FLAG_SORT_CHECK.  Results are invalid while a fault is injected; the
 * context stays usable once the hook is reset with (0, -1, 0). */
int cnb_ctx_inject_sort_faults(cnb_ctx *ctx, int32_t wait_limit, int64_t withheld_tile,
                               int64_t near_dest_bias);

/* No counterpart in the reference.  Sort mode of a context (default
 * CNB_SORT_FULL).  CNB_SORT_ADAPTIVE: cnb_sort_pairs with idx_in == NULL and
 * keys_in != keys_out first tries the near-sorted path -- keys that break
 * the ascending order (at every descent the shorter of the out-of-order runs
 * on its two sides, repeated in 4096-key windows until what is left ascends)
 * and keys outside the running max / min of the rest are taken out, sorted,
 * and merged back -- and runs the
 * full radix sort only when more than CNB_SORT_NEAR_CAP keys had to be
 * taken out.  Both paths return the same stable argsort; the choice is made
 * on the device (no synchronisation).  When the stream is being captured into
 * a CUDA graph, the full sort goes into a conditional node that the
 * near-sorted path switches off when it produced the result.  Bodies that
 * were sorted by their keys one step earlier mostly keep their order. */
#define CNB_SORT_FULL 0
#define CNB_SORT_ADAPTIVE 1
#define CNB_SORT_NEAR_CAP 2048
int cnb_ctx_set_sort_mode(cnb_ctx *ctx, int mode);

/* No counterpart in the reference.  out[0] = sorts of this context that took
 * the near-sorted path, out[1] = sorts that ran the full radix sort (host
 * array of 2; synchronises the device). */
int cnb_ctx_sort_stats(cnb_ctx *ctx, int64_t *out);

/* No counterpart in the reference: ORs the flags the context's kernels
 * raised into the caller's device status word and clears them (stream
 * ordered, no synchronisation). */
int cnb_ctx_take_flags(cnb_ctx *ctx, int32_t *status, void *stream);

/* No counterpart in the reference.  A stable (key, index) sort with output
 * identical to cnb_sort_pairs', for callers that cannot allocate device memory (a plugin
 * whose host application owns all device memory through its own pool, or
 * code running where a cudaMalloc and the synchronisation it may bring are
 * not allowed).  It takes no context and allocates nothing: its scratch is a
 * fixed device array inside libcnb.so, sized for at most
 * CNB_NOALLOC_MAX_KEYS keys (about 24.3 MiB, held on every GPU that loads the
 * library until the process exits).  Larger n returns CNB_E_TOO_LARGE.  It
 * runs the reduce-then-scan radix sort: three launches per 8-bit digit (24
 * for 63-bit keys, 12 for 30-bit keys) where cnb_sort_pairs runs one.  The
 * first call on a device looks up the array's device address and keeps it
 * for the life of the process (so make that call before any stream capture;
 * a cudaDeviceReset after it is not supported).  All calls share the array:
 * calls that overlap on the GPU race.  Buffer rules as for cnb_sort_pairs. */
#define CNB_NOALLOC_MAX_KEYS (1 << 20)
int cnb_sort_pairs_noalloc(const uint64_t *keys_in, uint64_t *keys_out, const uint32_t *idx_in,
                           uint32_t *perm_out, int64_t n, int key_bits, void *stream);

/* src/core/state.py:37-40 `a[sort_idx]` gathers: dst[k][i] = src[k][perm[i]]
 * for k < n_arrays (at most 8 float32 arrays). */
int cnb_gather_f32(const uint32_t *perm, int n_arrays, const float *const *src,
                   float *const *dst, int64_t n, void *stream);

/* src/kernels/tree_kernels.py:236-262 reset_tree_buffers(child, parent, counters, root_idx). */
int cnb_reset_tree_buffers(int32_t *child, int32_t *parent, int32_t *counters,
                           int32_t *root_idx, int64_t n_nodes, void *stream);

/* src/kernels/tree_kernels.py:60-129 build_tree(codes, children, parents). */
int cnb_build_tree(const uint64_t *codes, int32_t *children, int32_t *parents, int64_t n,
                   void *stream);

/* Topology check (no reference counterpart): every node but one root is the
 * child of exactly one internal node and parents[] agrees with children[];
 * otherwise CNB_FLAG_BAD_TOPOLOGY is set in status.  scratch: device int32
 * [2N] (overwritten). */
int cnb_validate_tree(const int32_t *children, const int32_t *parents, int64_t n,
                      int32_t *scratch, int32_t *status, void *stream);

/* src/kernels/tree_kernels.py:131-191 compute_multipoles(pos_x, pos_y, pos_z, mass,
 * children, parents, n_mass, n_com, n_min, n_max, counts).  n = bodies. */
int cnb_compute_multipoles(const float *px, const float *py, const float *pz,
                           const float *mass, const int32_t *children, const int32_t *parents,
                           float *n_mass, float *n_com, float *n_min, float *n_max,
                           int32_t *counts, int64_t n, int32_t *status, void *stream);

/* Extended upward pass (no reference counterpart beyond tree_kernels.py:131-214):
 * mode CNB_UPWARD_PLAIN reproduces compute_multipoles + normalize_com bit for
 * bit; CNB_UPWARD_COMPENSATED carries a two-sum error term with every float32
 * mass-weighted sum and sets the root's mass and CoM from a float64 reduction.
 * Writes the normalised n_com.  n_err ([M,4] float32, 16-byte aligned) holds
 * the compensation terms (compensated mode only, else may be NULL).
 * root_f64 (device, 4 doubles: mass, CoM x, y, z; required in compensated
 * mode, optional in plain mode, where the float32 tree is left untouched)
 * receives the float64 root values.  counts must be zero on entry. */
int cnb_upward(const float *px, const float *py, const float *pz, const float *mass,
               const int32_t *children, const int32_t *parents, float *n_mass, float *n_com,
               float *n_min, float *n_max, float *n_err, int32_t *counts, int64_t n, int mode,
               double *root_f64, int32_t *status, void *stream);

/* tree_kernels.py:131-214 compute_multipoles + normalize_com for the grouped
 * traversal: one pass that forms every node (float32 left + right sums,
 * Numba min/max, CoM normalised in float64 -- the reference's arithmetic)
 * and writes its record into node_table (the layout of cnb_pack_nodes,
 * bit-identical to cnb_upward + cnb_pack_nodes).  sums: scratch float32
 * [n_nodes, 4], 16-byte aligned (raw mass-weighted sums).  counts must be
 * zero on entry.  The reference-layout arrays are not written; get them
 * with cnb_unpack_nodes. */
int cnb_upward_table(const float *px, const float *py, const float *pz, const float *mass,
                     const int32_t *children, const int32_t *parents, int32_t *counts,
                     float *node_table, float *sums, int64_t n, int32_t *status, void *stream);

/* Reference-layout n_mass, n_com (normalised), n_min, n_max from a node table
 * (src/core/octree.py:85-93 get_buffers). */
int cnb_unpack_nodes(const float *node_table, float *n_mass, float *n_com, float *n_min,
                     float *n_max, int64_t n_nodes, void *stream);

/* src/kernels/tree_kernels.py:193-214 normalize_com(n_mass, n_com, n_nodes). */
int cnb_normalize_com(const float *n_mass, float *n_com, int64_t n_nodes, void *stream);

/* src/kernels/tree_kernels.py:216-234 find_root(parents, root_idx). */
int cnb_find_root(const int32_t *parents, int32_t *root_idx, int64_t n_nodes, void *stream);

/* src/kernels/tree_kernels.py:264-313 build_top_tree_cache(child, root_idx, top_nodes,
 * node_to_cache, cache_size).  node_to_cache must hold -1 for uncached nodes
 * on entry (src/core/engine.py:81 fills it). */
int cnb_build_top_tree_cache(const int32_t *child, const int32_t *root_idx,
                             int32_t *top_nodes, int32_t *node_to_cache, int32_t cache_size,
                             void *stream);

/* src/kernels/physics_kernels.py:14-153 compute_forces(pos_x, pos_y, pos_z, children,
 * n_mass, n_com, n_min, n_max, force, theta, G, soft, box, root, top_nodes,
 * node_to_cache, off): per-particle stack traversal for targets
 * off .. off+count-1 (n = bodies).  The top-tree cache only mirrors node data
 * and is not needed.  precision: CNB_PREC_F64 follows the reference's
 * float64 arithmetic, CNB_PREC_F32 computes in float32. */
int cnb_compute_forces(const float *px, const float *py, const float *pz,
                       const int32_t *children, const float *n_mass, const float *n_com,
                       const float *n_min, const float *n_max, float *force, double theta,
                       double G, double soft, double box, const int32_t *root_idx, int64_t off,
                       int64_t count, int64_t n, int precision, int32_t *status, void *stream);

/* src/kernels/physics_kernels.py:155-203 integrate(pos_x, pos_y, pos_z, vel_x, vel_y,
 * vel_z, force, a, H, dt). */
int cnb_integrate(float *px, float *py, float *pz, float *vx, float *vy, float *vz,
                  const float *force, int64_t n, double a, double H, double dt, void *stream);

/* src/kernels/render_kernels.py:12-47 render_density(pos_x, pos_y, pos_z, grid, mvp, res):
 * grid is [height, width] float32 (width == height == res in the reference),
 * mvp is a device float32[4,4]. */
int cnb_render_density(const float *px, const float *py, const float *pz, float *grid,
                       const float *mvp, int64_t n, int width, int height, void *stream);

/* src/kernels/tree_kernels.py:60-129 build_tree plus the index range
 * [lo, hi] of every internal node's bodies: ranges is int32 [N-1, 2]
 * (internal node N+i -> ranges[i]), 8-byte aligned.  Same children/parents
 * as cnb_build_tree. */
int cnb_build_tree_ranges(const uint64_t *codes, int32_t *children, int32_t *parents,
                          int32_t *ranges, int64_t n, void *stream);

/* Bucket table for cnb_forces_grouped (no reference counterpart): the
 * maximal subtrees holding at most max_size bodies.  workspace (device,
 * 16-byte aligned) is int32 [4 + 4N]: [0] bucket count, [1] work counter,
 * [2] deepest node stack seen by the traversal (entries; for CNB_MAC_REF_X
 * words of its stack region, one per whole-bucket entry and three per
 * part-bucket entry: 864 words in the main pass, 2048 for theta < 0.4, 4096
 * when a bucket is walked again), [3] the bodies' (index + 1)
 * summed over all buckets modulo 2^32 (N(N+1)/2 when the buckets tile the
 * bodies once; cnb_upward_table_buckets flags CNB_FLAG_BAD_TOPOLOGY
 * otherwise, and also when a bucket's nodes do not form a tree over its
 * bodies: the reference's tie rule for equal keys can leave a node without a
 * parent), then one
 * (first body, count, subtree node, 0) record per bucket. */
int cnb_make_buckets(const int32_t *ranges, const int32_t *parents, int64_t n, int max_size,
                     int32_t *workspace, void *stream);

/* cnb_build_tree_ranges, cnb_make_buckets (max_size) and cnb_find_root in
 * one launch, for the grouped step: also zeroes the internal nodes' climb
 * counters (counters int32 [2N-1]) and, when super_ws is not NULL, makes the
 * super-bucket table of cnb_forces_two_level (super_size bodies) there.  The
 * root is always node N (leaf 0 for N = 1).  Writes no leaf's children and
 * not the root's parent: those must hold -1 from an earlier
 * cnb_reset_tree_buffers (or the allocation).  Bucket tables list the same
 * buckets as cnb_make_buckets, in another order. */
int cnb_build_tree_buckets(const uint64_t *codes, int32_t *children, int32_t *parents,
                           int32_t *ranges, int32_t *counters, int32_t *root_idx, int64_t n,
                           int max_size, int32_t *workspace, int super_size, int32_t *super_ws,
                           void *stream);

/* cnb_make_buckets for several boxes in one tree (keys of
 * cnb_compute_codes_boxes): no bucket spans two boxes. */
int cnb_make_buckets_boxes(const int32_t *ranges, const int32_t *parents, const uint64_t *codes,
                           int box_bits, int64_t n, int max_size, int32_t *workspace,
                           void *stream);

/* Node table for cnb_forces_grouped: float32 [4, n_nodes, 4], 16-byte
 * aligned: 32-byte records (com x, y, z, mass | x-extent, 3-D extent,
 * child0 bits, child1 bits) for every node, then the boxes (min | max).
 * Built from the reference-layout tree (normalised n_com). */
int cnb_pack_nodes(const float *n_mass, const float *n_com, const float *n_min,
                   const float *n_max, const int32_t *children, float *node_table,
                   int64_t n_nodes, void *stream);

/* The B200 form of src/kernels/physics_kernels.py:14-153: one warp per
 * bucket of cnb_make_buckets (at most 32 * bodies_per_lane bodies, buckets
 * handed out by an atomic work counter), shared-memory node stack and
 * interaction list, float32 with rsqrt, the minimum image per pair only
 * where a bucket's bodies can see different images.  theta_per_bucket
 * (device float per bucket slot, may be NULL) overrides theta.  mac:
 * CNB_MAC_REF_X (each body gets exactly the nodes the reference's per-body
 * walk applies: the opening test is decided per body wherever the bucket's
 * box cannot decide it for all, in float64 where float32 rounding could
 * change it), CNB_MAC_REF_X_BUCKET or CNB_MAC_PERIODIC; forces are float32
 * sums.  For CNB_MAC_REF_X the reference's 64-entry stack limit
 * (physics_kernels.py:143-149, children silently dropped) is not
 * reproduced: it binds only on trees deeper than about 63 levels.
 * bodies_per_lane: 1 or 2 (buckets of
 * up to 32 or 64 bodies); block_warps: 2, 4 or 8 warps per block.  slab_mass
 * (CNB_MAC_PERIODIC only): nodes whose image differs between a bucket's
 * bodies are opened unless their mass is at most slab_mass, in which case
 * they are applied with the per-pair minimum image of their CoM (0 = exact
 * minimum-image semantics).  stats (device, 3 x uint64, may be NULL)
 * accumulates [body-node interactions, node tests, interactions applied
 * with the per-pair minimum image]. */
int cnb_forces_grouped(const float *px, const float *py, const float *pz,
                       const float *node_table, int32_t *workspace, float *force, int64_t n,
                       double theta, const float *theta_per_bucket, int mac, int bodies_per_lane,
                       int block_warps, double G, double soft, double box, double slab_mass,
                       unsigned long long *stats, int32_t *status, void *stream);

/* With CNB_MAC_REF_X the traversal runs in two passes: the main pass gives up
 * on a bucket whose node stacks would outgrow its shared-memory region (it
 * marks the bucket record's fourth word and writes no force for it), and a
 * second pass walks only the marked buckets again with a region 4.7 times as
 * large (two passes with the same nodes: the same forces).  Tests only:
 * cnb_exact_test_spill(k) makes the main pass give up on every k-th bucket
 * slot after its first round (0 = off; process-wide, not thread-safe). */
int cnb_exact_test_spill(int every);

/* Two-level form of cnb_forces_grouped (no reference counterpart; same
 * results as the one-level walk with the same mac, CNB_MAC_REF_X or
 * CNB_MAC_REF_X_BUCKET, up to float32 summation order).  The tree is cut
 * into super-buckets (maximal subtrees of at most super_bodies bodies, >= 32);
 * one warp per super-bucket walks the top of the tree once and keeps the
 * nodes every bucket inside it accepts (applied by each bucket from that
 * list) and the nodes only a bucket can decide (each bucket's walk starts
 * there).  ranges / parents: cnb_build_tree_ranges, from which the
 * super-bucket table is made in super_ws; both NULL: super_ws already holds
 * it (cnb_build_tree_buckets with the same super_bodies); workspace: the
 * bucket table of cnb_make_buckets; super_ws: device scratch of super_ws_bytes
 * (16-byte aligned), cnb_two_level_workspace_bytes recommends a size; a
 * super-bucket whose lists do not fit there walks from the root. */
int64_t cnb_two_level_workspace_bytes(int64_t n, int super_bodies);
int cnb_forces_two_level(const float *px, const float *py, const float *pz,
                         const float *node_table, const int32_t *ranges, const int32_t *parents,
                         int32_t *workspace, void *super_ws, int64_t super_ws_bytes,
                         int super_bodies, float *force, int64_t n, double theta, int mac,
                         int bodies_per_lane, int block_warps, double G, double soft, double box,
                         unsigned long long *stats, int32_t *status, void *stream);

/* ---- periodic (Ewald) force law (no reference counterpart; the reference
 * applies the minimum-image force of physics_kernels.py:118-141) ----
 * Unit box, d = source - target: the acceleration towards a point mass and
 * all its images (neutralising background) is f_per(d) = d/|d|^3 -
 * (4 pi/3) d + g(d), g smooth and O(|d|^3).
 *
 * Tabulates g, its Jacobian and its second derivatives on the octant
 * [0, 1/2]^3, (nt + 1)^3 points of spacing 1/(2 nt), computed in float64:
 * table is float32 [(nt + 1)^3, 24] (16-byte aligned), 2 <= nt <= 512. */
int cnb_ewald_table(float *table, int nt, void *stream);

/* cnb_forces_grouped under the periodic law: nodes open on their 3-D extent
 * (l^2 < theta^2 dmin^2), one image of every accepted node serves the whole
 * bucket, each body gets the softened monopoles plus, for every accepted
 * node, -(4 pi/3) m (c - x) + m g(c - centre) + m J(c - centre) (centre - x)
 * with g, J from the table of cnb_ewald_table.  quad (may be NULL): the
 * second central moments of cnb_upward_table_quad; accepted internal nodes
 * then also apply their quadrupole term, (15/2)(d.M d) d/r^7 - 3 M d/r^5 -
 * (3/2) tr(M) d/r^5, plus its periodic part (1/2) H(c - centre) : M from
 * the table's second derivatives of g (stats[2] then counts those
 * quadrupole interactions).  bucket_inter (device int32 per bucket slot, may
 * be NULL) receives the interactions each body of the bucket received: the
 * per-bucket cost the learned controller's labels weigh.  bucket_order (may
 * be NULL: slot order) is the order buckets are handed out in
 * (cnb_order_buckets). */
int cnb_forces_grouped_ewald(const float *px, const float *py, const float *pz,
                             const float *node_table, int32_t *workspace, float *force, int64_t n,
                             double theta, const float *theta_per_bucket, int bodies_per_lane,
                             int block_warps, double G, double soft, const float *ewald_table,
                             int ewald_nt, const float *quad, const int32_t *bucket_order,
                             int32_t *bucket_inter, unsigned long long *stats, int32_t *status,
                             void *stream);

/* No counterpart in the reference.  The order in which the grouped
 * traversal should take the buckets of a per-bucket theta (the bucket_order
 * input of cnb_forces_grouped_ewald): smallest theta, the most work, first,
 * in 32 bins over [0.2, 1.0], so that the persistent launch does not end on
 * a few expensive buckets.  order: device int32 per bucket slot. */
int cnb_order_buckets(const float *theta_per_bucket, const int32_t *workspace, int32_t *order,
                      void *stream);

/* cnb_upward_table that also forms the second central moment of every
 * internal node about its CoM (parallel-axis rule over the two children):
 * quad is float32 [2 * n_nodes, 4] (16-byte aligned), node v at rows 2v,
 * 2v+1: (xx, xy, xz, yy), (yz, zz, 0, 0); leaf rows are not written.  The
 * node table's 3-D-extent slot then holds b_max, the largest distance from
 * the node's CoM to a corner of its box, which the periodic-law opening test
 * uses as the node's size. */
int cnb_upward_table_quad(const float *px, const float *py, const float *pz, const float *mass,
                          const int32_t *children, const int32_t *parents, int32_t *counts,
                          float *node_table, float *sums, float *quad, int64_t n,
                          int32_t *status, void *stream);

/* cnb_upward_table (quad NULL) or cnb_upward_table_quad, computed over the
 * bucket table of cnb_make_buckets (buckets of at most 64 bodies; larger
 * ones raise CNB_FLAG_LIST_OVERFLOW): one warp per bucket forms the nodes
 * inside it with shared-memory counters, then one thread per bucket root
 * climbs the levels above.  Same table, bit for bit; sums (climb scratch)
 * then holds raw sums only for bucket roots and the nodes above them. */
int cnb_upward_table_buckets(const float *px, const float *py, const float *pz, const float *mass,
                             const int32_t *children, const int32_t *parents,
                             const int32_t *workspace, int32_t *counts, float *node_table,
                             float *sums, float *quad, int64_t n, int32_t *status, void *stream);

/* cnb_forces_grouped_boxes under the periodic law of cnb_forces_grouped_ewald:
 * every box is periodic on its own unit cube (bucket_inter as there). */
int cnb_forces_grouped_boxes_ewald(const float *px, const float *py, const float *pz,
                                   const float *node_table, int32_t *workspace, float *force,
                                   int64_t n, const uint64_t *codes, int box_bits,
                                   const int32_t *box_roots, const float *box_params,
                                   const float *theta_per_bucket, int bodies_per_lane,
                                   int block_warps, double G, const float *ewald_table,
                                   int ewald_nt, int32_t *bucket_inter,
                                   unsigned long long *stats, int32_t *status, void *stream);

/* Float64 periodic direct sum for the bodies listed in targets (accuracy
 * oracle of the periodic law): per pair the softened monopole at the minimum
 * image plus f_per - d/|d|^3, with the Ewald sums carried to float64
 * precision.  out is float64 [n_targets, 3]. */
int cnb_direct_sum_ewald_f64(const float *px, const float *py, const float *pz,
                             const float *mass, int64_t n, const int64_t *targets,
                             int64_t n_targets, double G, double soft, double *out, void *stream);

/* src/utils/visualizer.py:115-171 colorize_frame (+ the 8-bit packing of
 * src/core/engine.py:139): grid [height, width] float32 -> rgb float32
 * [height, width, 3] and/or rgb8 uint8 [height, width, 3] (either may be
 * NULL).  scratch: one device uint32 (the running maximum). */
int cnb_colorize(const float *grid, int width, int height, float *rgb, unsigned char *rgb8,
                 unsigned int *scratch, void *stream);

/* ---- many independent boxes in one launch (no reference counterpart) ----
 * Keys carry the box id in their top bits: key = box << 3L | morton_L(x,y,z),
 * L = (63 - box_bits) / 3 bits per axis, coordinates in each box's own unit
 * cube.  One sort and one Karras build then make every box one subtree. */
int cnb_compute_codes_boxes(const float *x, const float *y, const float *z, const int32_t *box,
                            uint64_t *codes, int64_t n, int box_bits, void *stream);

/* Subtree root of every box (int32 [n_boxes], -1 for an empty box) from the
 * sorted box keys and the tree of cnb_build_tree_ranges. */
int cnb_box_roots(const int32_t *ranges, const int32_t *parents, const uint64_t *codes,
                  int box_bits, int64_t n, int n_boxes, int32_t *roots, void *stream);

/* cnb_forces_grouped over many boxes: every bucket walks its own box's
 * subtree with its box's (theta, softening, slab mass, unused) from
 * box_params (float32 [n_boxes, 4], 16-byte aligned); theta_per_bucket, if
 * given, overrides theta.  Each box is periodic on its own unit cube. */
int cnb_forces_grouped_boxes(const float *px, const float *py, const float *pz,
                             const float *node_table, int32_t *workspace, float *force, int64_t n,
                             const uint64_t *codes, int box_bits, const int32_t *box_roots,
                             const float *box_params, const float *theta_per_bucket, int mac,
                             int bodies_per_lane, int block_warps, double G,
                             unsigned long long *stats,
                             int32_t *status, void *stream);

/* physics_kernels.py:155-203 integrate with per-box (a, H, dt): box_aHdt is
 * float64 [n_boxes, 3] on the device, so a captured step can advance it. */
int cnb_integrate_boxes(float *px, float *py, float *pz, float *vx, float *vy, float *vz,
                        const float *force, const uint64_t *codes, int box_bits, int64_t n,
                        const double *box_aHdt, void *stream);

/* ---- learned opening-angle controller (no reference counterpart) ----
 * An MLP 12 -> 64 -> 64 -> 1 (SiLU) maps features of a bucket to its theta
 * in [0.2, 1.0].  Parameters: CNB_MLP_PARAMS float32 values, in the order
 * W1[64][12], b1[64], W2[64][64], b2[64], w3[64], b3. */
#define CNB_MLP_PARAMS 5057

/* 12 features per bucket (float32 [buckets, 12]) from the node table,
 * parents and the bucket table of cnb_make_buckets; at most max_buckets.
 * accel (float32 [N, 3], required) holds the bodies' accelerations of the
 * previous step; perm (may be NULL: identity) maps each body's current
 * position in the sorted order to its row of accel (the sort's
 * permutation).  One feature is the bucket's mean |a| over the local force
 * scale G M / l^2 of its third ancestor. */
int cnb_bucket_features(const float *node_table, const int32_t *parents,
                        const int32_t *workspace, int64_t n, const float *accel,
                        const uint32_t *perm, float *features, int max_buckets, void *stream);

/* Fused inference: features and the network (bfloat16 weights, float32
 * accumulation; the 64 x 64 layer on the tensor cores with the first layer's
 * outputs rounded to bfloat16) -> theta per bucket slot, the
 * theta_per_bucket input of cnb_forces_grouped (accel, perm as for
 * cnb_bucket_features). */
int cnb_controller_theta(const float *node_table, const int32_t *parents,
                         const int32_t *workspace, int64_t n, const float *accel,
                         const uint32_t *perm, const void *weights_bf16, float *theta,
                         int max_buckets, void *stream);

/* The network on given features with float32 weights. */
int cnb_mlp_predict(const float *features, int n, const float *weights, float *theta,
                    void *stream);

/* Training: loss = mean over samples of c (theta - label)^2, c = over_weight
 * where theta > label, else 1; writes the gradient (CNB_MLP_PARAMS floats)
 * and the loss.  scratch: float32 [4 * 64 * n + n]. */
int cnb_mlp_grad(const float *features, const float *labels, int n, const float *weights,
                 float over_weight, float *scratch, float *grad, float *loss, void *stream);

/* cnb_mlp_grad with the three 64-wide contractions on the tensor cores
 * (mma.sync m16n8k16, bfloat16 operands, float32 accumulation): the forward
 * second layer, the backward dH1 = dA2 W2 and the parameter gradients dW2 =
 * dA2^T H1 and dW1 = dA1^T X over the samples; layer 1, the activations'
 * derivatives, the loss, the bias sums and dw3 stay in float32.  scratch:
 * device, 16-byte aligned, at least cnb_mlp_grad_mma_scratch_bytes(n)
 * bytes (bfloat16 activations, transposed). */
int64_t cnb_mlp_grad_mma_scratch_bytes(int n);
int cnb_mlp_grad_mma(const float *features, const float *labels, int n, const float *weights,
                     float over_weight, void *scratch, int64_t scratch_bytes, float *grad,
                     float *loss, void *stream);

/* One Adam update of n parameters (step t >= 1). */
int cnb_adam_step(float *params, const float *grad, float *m, float *v, int n, float lr,
                  float beta1, float beta2, float eps, int t, void *stream);

/* float32 -> bfloat16 (round to nearest even). */
int cnb_to_bf16(const float *src, void *dst, int n, void *stream);

/* Float64 minimum-image direct sum (the force law of
 * src/kernels/physics_kernels.py:118-141 over every pair) for the bodies
 * listed in targets (device int64[n_targets]); out is float64 [n_targets,3].
 * Accuracy reference for the tree forces and labels for the learned
 * opening-angle controller. */
int cnb_direct_sum_f64(const float *px, const float *py, const float *pz, const float *mass,
                       int64_t n, const int64_t *targets, int64_t n_targets, double G,
                       double soft, double *out, void *stream);

/* FP32 FMA throughput probe (no reference counterpart): `blocks` x 256
 * threads, 16 * iters flops per thread; out holds blocks*256 floats. */
int cnb_fma_probe(float *out, int64_t iters, int blocks, void *stream);
/* The same with packed float2 FMAs (FFMA2): 32 flops per thread per iteration. */
int cnb_fma2_probe(float *out, int64_t iters, int blocks, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* CNB_H */
