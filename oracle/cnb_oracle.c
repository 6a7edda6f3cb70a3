/*
 * cnb_oracle.c -- CPU restatement of Cosmo-NBody's Barnes-Hut step.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA library
 * (libcnb.so): tests, the smoke check and the CPU-baseline leg of bench.py
 * call it; the product path never does.
 *
 * Every function restates one reference kernel, keeping the arithmetic
 * types that compiled Numba gives the reference source (float32 array
 * elements, Python-float scalars and `round()`/`1.0 /` promoting to
 * float64).  Each function cites the reference file:line it follows.
 *
 * Pinning: integer stages are compared bit-exactly, and float stages by
 * tolerance, against the reference kernels themselves executed under
 * Numba's CUDA simulator (fixtures in tests/golden/, generated by
 * tests/golden/make_golden.py).
 *
 * Build: oracle/build_oracle.sh (gcc -O2 -fopenmp, no fast-math, no FMA
 * contraction, so float64 results are IEEE round-to-nearest per operation).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------ */
/* Morton keys                                                         */
/* ------------------------------------------------------------------ */

/* src/kernels/morton.py:13-37 -- the reference's masks keep only the low
 * 10 bits of the input: (v|v<<16)&0x030000FF ... &0x09249249. */
static uint64_t spread_ref(uint64_t v) {
    v = (v | (v << 16)) & 0x030000FFull;
    v = (v | (v << 8)) & 0x0300F00Full;
    v = (v | (v << 4)) & 0x030C30C3ull;
    v = (v | (v << 2)) & 0x09249249ull;
    return v;
}

/* Full 21-bit interleave written bit by bit (independent of any mask
 * trick), for the corrected 63-bit key the reference's docstring
 * describes (morton.py:40-53). */
static uint64_t spread21_loop(uint64_t v) {
    uint64_t r = 0;
    for (int b = 0; b < 21; ++b) r |= ((v >> b) & 1ull) << (3 * b);
    return r;
}

/* morton.py:57-59: ix = uint64(x * 2097152.0), x float32 promoted to
 * float64 (exact, power-of-two scale), truncation toward zero.  Negative
 * and NaN inputs are undefined in the reference; here they map to 0. */
static uint64_t scale21(float x) {
    double s = (double)x * 2097152.0;
    if (!(s > 0.0)) return 0;
    if (s >= 18446744073709551615.0) return ~0ull;
    return (uint64_t)s;
}

/* morton.py:40-63 (mode 0, reference-exact 30-bit keys) and the corrected
 * 63-bit key (mode 1: coordinates clamped to [0, 2^21-1]). */
uint64_t orc_morton(float x, float y, float z, int mode) {
    uint64_t ix = scale21(x), iy = scale21(y), iz = scale21(z);
    if (mode == 0) return spread_ref(ix) | (spread_ref(iy) << 1) | (spread_ref(iz) << 2);
    const uint64_t lim = (1ull << 21) - 1;
    if (ix > lim) ix = lim;
    if (iy > lim) iy = lim;
    if (iz > lim) iz = lim;
    return spread21_loop(ix) | (spread21_loop(iy) << 1) | (spread21_loop(iz) << 2);
}

/* morton.py:65-90 compute_codes: codes[i] = key, indices[i] = i. */
void orc_compute_codes(const float *x, const float *y, const float *z, uint64_t *codes,
                       uint32_t *indices, int64_t n, int mode) {
    for (int64_t i = 0; i < n; ++i) {
        codes[i] = orc_morton(x[i], y[i], z[i], mode);
        if (indices) indices[i] = (uint32_t)i;
    }
}

/* state.py:35 `cp.argsort(codes)`: a stable ascending argsort (ties keep
 * index order).  LSD radix sort on 8-bit digits, 8 passes, skipping digits
 * that are constant over the input. */
void orc_argsort_stable(const uint64_t *keys, int64_t n, int64_t *perm) {
    int64_t *tmp = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
    int64_t *a = perm, *b = tmp;
    for (int64_t i = 0; i < n; ++i) a[i] = i;
    for (int pass = 0; pass < 8; ++pass) {
        int shift = 8 * pass;
        int64_t cnt[257];
        memset(cnt, 0, sizeof(cnt));
        for (int64_t i = 0; i < n; ++i) cnt[((keys[a[i]] >> shift) & 255) + 1]++;
        int constant = 0;
        for (int d = 0; d < 256; ++d) if (cnt[d + 1] == n) constant = 1;
        if (constant) continue;
        for (int d = 0; d < 256; ++d) cnt[d + 1] += cnt[d];
        for (int64_t i = 0; i < n; ++i) b[cnt[(keys[a[i]] >> shift) & 255]++] = a[i];
        int64_t *t = a; a = b; b = t;
    }
    if (a != perm) memcpy(perm, a, sizeof(int64_t) * (size_t)n);
    free(tmp);
}

/* ------------------------------------------------------------------ */
/* Tree                                                                */
/* ------------------------------------------------------------------ */

/* tree_kernels.py:236-262 reset_tree_buffers. */
void orc_reset_tree(int32_t *child, int32_t *parent, int32_t *counters, int32_t *root_idx,
                    int64_t m) {
    if (root_idx) root_idx[0] = 0;
    for (int64_t i = 0; i < m; ++i) {
        child[2 * i] = -1;
        child[2 * i + 1] = -1;
        parent[i] = -1;
        counters[i] = 0;
    }
}

/* tree_kernels.py:17-34 clz64 (software count of leading zeros). */
static int clz64(uint64_t v) {
    if (v == 0) return 64;
    int n = 0;
    if ((v & 0xFFFFFFFF00000000ull) == 0) { n += 32; v <<= 32; }
    if ((v & 0xFFFF000000000000ull) == 0) { n += 16; v <<= 16; }
    if ((v & 0xFF00000000000000ull) == 0) { n += 8; v <<= 8; }
    if ((v & 0xF000000000000000ull) == 0) { n += 4; v <<= 4; }
    if ((v & 0xC000000000000000ull) == 0) { n += 2; v <<= 2; }
    if ((v & 0x8000000000000000ull) == 0) { n += 1; }
    return n;
}

/* tree_kernels.py:36-58 delta_fn.  Equal keys use 64 + (63 - clz64(i^j)),
 * i.e. 64 + the index of the highest set bit of i^j (the reference's own
 * tie rule, kept as is). */
static int64_t delta_fn(const uint64_t *codes, int64_t i, int64_t j, int64_t n) {
    if (j < 0 || j >= n) return -1;
    if (codes[i] == codes[j]) return 64 + (63 - clz64((uint64_t)(i ^ j)));
    return clz64(codes[i] ^ codes[j]);
}

/* tree_kernels.py:60-129 build_tree (Karras 2012). */
void orc_build_tree(const uint64_t *codes, int32_t *children, int32_t *parents, int64_t n) {
    for (int64_t i = 0; i < n - 1; ++i) {
        int64_t idx = i + n;
        int64_t d_prev = delta_fn(codes, i, i - 1, n);
        int64_t d_next = delta_fn(codes, i, i + 1, n);
        int64_t dir = d_next > d_prev ? 1 : -1;
        int64_t min_delta = d_next > d_prev ? d_prev : d_next;
        int64_t l_max = 2;
        while (delta_fn(codes, i, i + l_max * dir, n) > min_delta) l_max *= 2;
        int64_t l = 0;
        for (int64_t t = l_max / 2; t >= 1; t /= 2)
            if (delta_fn(codes, i, i + (l + t) * dir, n) > min_delta) l += t;
        int64_t j = i + l * dir;
        int64_t delta_node = delta_fn(codes, i, j, n);
        int64_t s = 0;
        for (int64_t t = l; t > 0;) {
            int64_t step = (t + 1) / 2;
            if (delta_fn(codes, i, i + (s + step) * dir, n) > delta_node) s += step;
            t -= step;
        }
        int64_t gamma = i + s * dir;
        if (dir == -1) gamma -= 1;
        int64_t left = gamma, right = gamma + 1;
        int64_t lo = i < j ? i : j, hi = i < j ? j : i;
        int32_t c0 = (int32_t)(lo == left ? left : left + n);
        int32_t c1 = (int32_t)(hi == right ? right : right + n);
        children[2 * idx] = c0;
        children[2 * idx + 1] = c1;
        parents[c0] = (int32_t)idx;
        parents[c1] = (int32_t)idx;
    }
}

/* Numba's min/max on two floats: min(a,b) = b if b < a else a
 * (numba/cpython/builtins.py do_minmax, used by tree_kernels.py:182-188). */
static float pmin(float a, float b) { return b < a ? b : a; }
static float pmax(float a, float b) { return b > a ? b : a; }

/* tree_kernels.py:131-191 compute_multipoles, run serially.  Each internal
 * node is formed once, as (left + right) in that order, by the second
 * arrival, so the serial run produces the same bits as any parallel
 * schedule.  Returns 0, or -1 if a climb exceeded m steps (cyclic
 * topology). */
int orc_compute_multipoles(const float *px, const float *py, const float *pz, const float *mass,
                           const int32_t *children, const int32_t *parents, float *n_mass,
                           float *n_com, float *n_min, float *n_max, int32_t *counts, int64_t n) {
    int64_t m = 2 * n - 1;
    int bad = 0;
    for (int64_t i = 0; i < n; ++i) {
        float mi = mass[i], x = px[i], y = py[i], z = pz[i];
        n_mass[i] = mi;
        n_com[3 * i] = x * mi;
        n_com[3 * i + 1] = y * mi;
        n_com[3 * i + 2] = z * mi;
        n_min[3 * i] = x; n_min[3 * i + 1] = y; n_min[3 * i + 2] = z;
        n_max[3 * i] = x; n_max[3 * i + 1] = y; n_max[3 * i + 2] = z;
        int64_t curr = i;
        for (int64_t guard = 0;; ++guard) {
            if (guard > m) { bad = 1; break; }
            int32_t p = parents[curr];
            if (p == -1) break;
            if (counts[p]++ == 0) break;
            int32_t l = children[2 * p], r = children[2 * p + 1];
            n_mass[p] = n_mass[l] + n_mass[r];
            for (int k = 0; k < 3; ++k) {
                n_com[3 * p + k] = n_com[3 * l + k] + n_com[3 * r + k];
                n_min[3 * p + k] = pmin(n_min[3 * l + k], n_min[3 * r + k]);
                n_max[3 * p + k] = pmax(n_max[3 * l + k], n_max[3 * r + k]);
            }
            curr = p;
        }
    }
    return bad ? -1 : 0;
}

/* tree_kernels.py:193-214 normalize_com: inv = 1.0 / m in float64, the
 * float32 com multiplied by it in float64 and stored back as float32. */
void orc_normalize_com(const float *n_mass, float *n_com, int64_t m) {
    for (int64_t i = 0; i < m; ++i) {
        if (n_mass[i] > 0) {
            double inv = 1.0 / (double)n_mass[i];
            for (int k = 0; k < 3; ++k) n_com[3 * i + k] = (float)((double)n_com[3 * i + k] * inv);
        }
    }
}

/* tree_kernels.py:216-234 find_root: a node whose parent is -1 (the
 * reference's atomic exchange keeps an arbitrary one if several exist;
 * here the highest index, which equals the reference for a valid tree). */
int32_t orc_find_root(const int32_t *parents, int64_t m) {
    int32_t root = 0;
    for (int64_t i = 0; i < m; ++i)
        if (parents[i] == -1) root = (int32_t)i;
    return root;
}

/* tree_kernels.py:264-313 build_top_tree_cache (breadth-first order). */
void orc_build_top_tree_cache(const int32_t *child, int32_t root, int32_t *top_nodes,
                              int32_t *node_to_cache, int32_t cache_size) {
    if (root == -1) return;
    top_nodes[0] = root;
    node_to_cache[root] = 0;
    int32_t rd = 0, wr = 1;
    while (rd < wr && wr < cache_size) {
        int32_t curr = top_nodes[rd];
        int32_t c1 = child[2 * curr];
        if (c1 != -1 && wr < cache_size) { top_nodes[wr] = c1; node_to_cache[c1] = wr; wr++; }
        int32_t c2 = child[2 * curr + 1];
        if (c2 != -1 && wr < cache_size) { top_nodes[wr] = c2; node_to_cache[c2] = wr; wr++; }
        rd++;
    }
    while (wr < cache_size) top_nodes[wr++] = -1;
}

/* ------------------------------------------------------------------ */
/* Forces                                                              */
/* ------------------------------------------------------------------ */

/* physics_kernels.py:14-153 compute_forces for one target.  Node data are
 * float32; `dx -= round(dx)` turns the displacement into float64 (round
 * returns int64), so d2, the opening test and the accumulation are
 * float64, as compiled Numba types them.  The stack holds 64 entries and
 * silently drops both children when fewer than two slots are free
 * (physics_kernels.py:143); *overflow counts those drops. */
static void force_one(const float *px, const float *py, const float *pz, const int32_t *children,
                      const float *n_mass, const float *n_com, const float *n_min,
                      const float *n_max, double theta, double G, double soft, double box,
                      int32_t root, int64_t i, double acc[3], int64_t *overflow,
                      int64_t *visits, int64_t *accepted) {
    float x = px[i], y = py[i], z = pz[i];
    double ax = 0.0, ay = 0.0, az = 0.0;
    int32_t stack[64];
    int top = 0;
    stack[top++] = root;
    double theta_sq = theta * theta;
    while (top > 0) {
        int32_t node = stack[--top];
        if (visits) (*visits)++;
        float nm = n_mass[node];
        float cx = n_com[3 * node], cy = n_com[3 * node + 1], cz = n_com[3 * node + 2];
        float mnx = n_min[3 * node], mxx = n_max[3 * node];
        int32_t c1 = children[2 * node], c2 = children[2 * node + 1];
        if (nm <= 0) continue;
        float dxf = cx - x, dyf = cy - y, dzf = cz - z;
        double dx = (double)dxf - (double)llrint((double)dxf);
        double dy = (double)dyf - (double)llrint((double)dyf);
        double dz = (double)dzf - (double)llrint((double)dzf);
        double d2 = dx * dx + dy * dy + dz * dz;
        int is_leaf = (c1 == -1);
        float sxf = mxx - mnx;
        double sx = ((double)sxf > box * 0.5) ? box : (double)sxf;
        int mac_pass = (sx * sx) < (theta_sq * d2);
        if (is_leaf || mac_pass) {
            if (accepted) (*accepted)++;
            if (d2 > 1e-7) {
                double d_inv = 1.0 / sqrt(d2 + soft * soft);
                double f = G * (double)nm * (d_inv * d_inv * d_inv);
                ax += f * dx;
                ay += f * dy;
                az += f * dz;
            }
        } else {
            if (top + 1 < 64) {
                if (c1 != -1) stack[top++] = c2;
                if (c2 != -1) stack[top++] = c1;
            } else if (overflow) {
                (*overflow)++;
            }
        }
    }
    acc[0] = ax;
    acc[1] = ay;
    acc[2] = az;
}

/* compute_forces over targets off .. off+count-1; force is [N,3] float32.
 * Returns the number of stack drops; *visits (optional) receives the total
 * number of popped nodes, *accepted_out (optional) the number of (body, node)
 * pairs the opening test accepted (leaves included, before the d2 cut). */
int64_t orc_compute_forces(const float *px, const float *py, const float *pz,
                           const int32_t *children, const float *n_mass, const float *n_com,
                           const float *n_min, const float *n_max, float *force, double theta,
                           double G, double soft, double box, int32_t root, int64_t off,
                           int64_t count, int nthreads, int64_t *visits_out,
                           int64_t *accepted_out) {
    int64_t overflow = 0, visits = 0, accepted = 0;
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads) reduction(+ : overflow, visits, accepted)
#endif
    for (int64_t t = 0; t < count; ++t) {
        double acc[3];
        int64_t i = off + t;
        force_one(px, py, pz, children, n_mass, n_com, n_min, n_max, theta, G, soft, box, root, i,
                  acc, &overflow, &visits, &accepted);
        force[3 * i] = (float)acc[0];
        force[3 * i + 1] = (float)acc[1];
        force[3 * i + 2] = (float)acc[2];
    }
    if (visits_out) *visits_out = visits;
    if (accepted_out) *accepted_out = accepted;
    return overflow;
}

/* Same traversal, float64 results for an explicit target list. */
int64_t orc_forces_targets_f64(const float *px, const float *py, const float *pz,
                               const int32_t *children, const float *n_mass, const float *n_com,
                               const float *n_min, const float *n_max, double theta, double G,
                               double soft, double box, int32_t root, const int64_t *targets,
                               int64_t nt, double *out, int nthreads) {
    int64_t overflow = 0;
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 16) num_threads(nthreads) reduction(+ : overflow)
#endif
    for (int64_t t = 0; t < nt; ++t)
        force_one(px, py, pz, children, n_mass, n_com, n_min, n_max, theta, G, soft, box, root,
                  targets[t], out + 3 * t, &overflow, NULL, NULL);
    return overflow;
}

/* Float64 minimum-image direct sum (the force law of
 * physics_kernels.py:118-141 applied to every pair, no tree):
 * a_i = sum_{j: d2 > 1e-7} G m_j d / (d2 + soft^2)^{3/2},
 * d = x_j - x_i - round(x_j - x_i) per axis, all in float64. */
void orc_direct_sum(const float *px, const float *py, const float *pz, const float *mass,
                    int64_t n, const int64_t *targets, int64_t nt, double G, double soft,
                    double *out, int nthreads) {
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads)
#endif
    for (int64_t t = 0; t < nt; ++t) {
        int64_t i = targets[t];
        double xi = px[i], yi = py[i], zi = pz[i];
        double ax = 0.0, ay = 0.0, az = 0.0, s2 = soft * soft;
        for (int64_t j = 0; j < n; ++j) {
            double dx = (double)px[j] - xi, dy = (double)py[j] - yi, dz = (double)pz[j] - zi;
            dx -= nearbyint(dx);
            dy -= nearbyint(dy);
            dz -= nearbyint(dz);
            double d2 = dx * dx + dy * dy + dz * dz;
            if (d2 > 1e-7) {
                double r = 1.0 / sqrt(d2 + s2);
                double f = G * (double)mass[j] * r * r * r;
                ax += f * dx;
                ay += f * dy;
                az += f * dz;
            }
        }
        out[3 * t] = ax;
        out[3 * t + 1] = ay;
        out[3 * t + 2] = az;
    }
}

/* ------------------------------------------------------------------ */
/* Integrator and splat                                                */
/* ------------------------------------------------------------------ */

/* physics_kernels.py:155-203 integrate: float64 kick with Hubble drag and
 * drift, periodic wrap by x - floor(x), stored as float32. */
void orc_integrate(float *px, float *py, float *pz, float *vx, float *vy, float *vz,
                   const float *force, int64_t n, double a, double H, double dt) {
    double drag = 1.0 - (H * dt);
    double f_scale = 1.0 / a;
    double drift = 1.0 / a;
    for (int64_t i = 0; i < n; ++i) {
        double v[3], p[3];
        float *vv[3] = {vx, vy, vz};
        float *pp[3] = {px, py, pz};
        for (int k = 0; k < 3; ++k) {
            v[k] = (double)vv[k][i] * drag + ((double)force[3 * i + k] * f_scale * dt);
            vv[k][i] = (float)v[k];
        }
        for (int k = 0; k < 3; ++k) {
            p[k] = (double)pp[k][i] + v[k] * dt * drift;
            p[k] = p[k] - floor(p[k]);
            pp[k][i] = (float)p[k];
        }
    }
}

/* render_kernels.py:12-47 render_density, generalised to a width x height
 * grid (width == height == res is the reference).  Clip coordinates are
 * float32 sums of float32 products (no fused multiply-add), 1.0 / w and the
 * screen mapping are float64, and 2.5 / w is added as float32.  Returns the
 * number of splatted particles; pix (optional) receives each particle's
 * flat pixel index or -1. */
int64_t orc_render_density(const float *px, const float *py, const float *pz, float *grid,
                           const float *mvp, int64_t n, int width, int height, int64_t *pix) {
    int64_t hits = 0;
    for (int64_t i = 0; i < n; ++i) {
        float x = px[i], y = py[i], z = pz[i];
        volatile float t0, t1, t2;
        t0 = mvp[0] * x; t1 = mvp[1] * y; t2 = mvp[2] * z;
        float xc = ((t0 + t1) + t2) + mvp[3];
        t0 = mvp[4] * x; t1 = mvp[5] * y; t2 = mvp[6] * z;
        float yc = ((t0 + t1) + t2) + mvp[7];
        t0 = mvp[12] * x; t1 = mvp[13] * y; t2 = mvp[14] * z;
        float wc = ((t0 + t1) + t2) + mvp[15];
        if (pix) pix[i] = -1;
        if ((double)wc > 0.01) {
            double inv = 1.0 / (double)wc;
            double sx = ((double)xc * inv + 1.0) * 0.5 * (double)width;
            double sy = (1.0 - (double)yc * inv) * 0.5 * (double)height;
            if (0 <= sx && sx < width && 0 <= sy && sy < height) {
                int64_t p = (int64_t)sy * width + (int64_t)sx;
                grid[p] += (float)(2.5 * inv);
                if (pix) pix[i] = p;
                hits++;
            }
        }
    }
    return hits;
}
