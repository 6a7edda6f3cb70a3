"""CPU oracle for the Barnes-Hut step -- TEST INFRASTRUCTURE ONLY.

numpy front end over ``oracle/liboracle.so`` (built from ``cnb_oracle.c`` by
``build_oracle.sh``).  Only tests, ``__graft_entry__.smoke()`` and the CPU
baseline leg of ``bench.py`` use it, as the checker; the product path
(``cnb``) never imports it.

Each wrapper restates one reference kernel of Cosmo-NBody (file:line in the
docstrings).  ``run_reference_step`` chains them the way
``src/core/engine.py:55-123`` does, with ``np.argsort(kind="stable")``
semantics for ``cp.argsort`` (``src/core/state.py:35``).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "liboracle.so")
_lib = None

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_i64 = C.c_int64
_d = C.c_double


def build():
    """Compile liboracle.so from cnb_oracle.c."""
    subprocess.run(["bash", os.path.join(_HERE, "build_oracle.sh")], check=True)


def lib():
    global _lib
    if _lib is not None:
        return _lib
    src = os.path.join(_HERE, "cnb_oracle.c")
    if not os.path.exists(_SO) or os.path.getmtime(_SO) < os.path.getmtime(src):
        build()
    L = C.CDLL(_SO)
    L.orc_morton.restype = C.c_uint64
    L.orc_morton.argtypes = [C.c_float, C.c_float, C.c_float, C.c_int]
    L.orc_compute_codes.argtypes = [_f32p, _f32p, _f32p, _u64p, _u32p, _i64, C.c_int]
    L.orc_argsort_stable.argtypes = [_u64p, _i64, _i64p]
    L.orc_reset_tree.argtypes = [_i32p, _i32p, _i32p, _i32p, _i64]
    L.orc_build_tree.argtypes = [_u64p, _i32p, _i32p, _i64]
    L.orc_compute_multipoles.restype = C.c_int
    L.orc_compute_multipoles.argtypes = [_f32p, _f32p, _f32p, _f32p, _i32p, _i32p, _f32p, _f32p,
                                         _f32p, _f32p, _i32p, _i64]
    L.orc_normalize_com.argtypes = [_f32p, _f32p, _i64]
    L.orc_find_root.restype = C.c_int32
    L.orc_find_root.argtypes = [_i32p, _i64]
    L.orc_build_top_tree_cache.argtypes = [_i32p, C.c_int32, _i32p, _i32p, C.c_int32]
    L.orc_compute_forces.restype = C.c_int64
    L.orc_compute_forces.argtypes = [_f32p, _f32p, _f32p, _i32p, _f32p, _f32p, _f32p, _f32p,
                                     _f32p, _d, _d, _d, _d, C.c_int32, _i64, _i64, C.c_int,
                                     C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    L.orc_forces_targets_f64.restype = C.c_int64
    L.orc_forces_targets_f64.argtypes = [_f32p, _f32p, _f32p, _i32p, _f32p, _f32p, _f32p, _f32p,
                                         _d, _d, _d, _d, C.c_int32, _i64p, _i64, _f64p, C.c_int]
    L.orc_direct_sum.argtypes = [_f32p, _f32p, _f32p, _f32p, _i64, _i64p, _i64, _d, _d, _f64p,
                                 C.c_int]
    L.orc_integrate.argtypes = [_f32p, _f32p, _f32p, _f32p, _f32p, _f32p, _f32p, _i64, _d, _d, _d]
    L.orc_render_density.restype = C.c_int64
    L.orc_render_density.argtypes = [_f32p, _f32p, _f32p, _f32p, _f32p, _i64, C.c_int, C.c_int,
                                     C.c_void_p]
    _lib = L
    return L


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


KEY_COMPAT30 = 0
KEY_MORTON63 = 1


def compute_codes(x, y, z, key_mode=KEY_COMPAT30):
    """src/kernels/morton.py:65-90 -> (codes uint64[N], indices uint32[N])."""
    x, y, z = _f32(x), _f32(y), _f32(z)
    n = x.size
    codes = np.zeros(n, np.uint64)
    idx = np.zeros(n, np.uint32)
    lib().orc_compute_codes(x, y, z, codes, idx, n, key_mode)
    return codes, idx


def argsort_stable(codes):
    """src/core/state.py:35 cp.argsort(codes), stable ascending."""
    codes = np.ascontiguousarray(codes, dtype=np.uint64)
    perm = np.zeros(codes.size, np.int64)
    lib().orc_argsort_stable(codes, codes.size, perm)
    return perm


def build_tree(codes):
    """tree_kernels.py:236-262 reset then tree_kernels.py:60-129 build_tree.
    Returns (children int32[M,2], parents int32[M])."""
    codes = np.ascontiguousarray(codes, dtype=np.uint64)
    n = codes.size
    m = max(2 * n - 1, 1)
    children = np.full((m, 2), -1, np.int32)
    parents = np.full(m, -1, np.int32)
    counters = np.zeros(m, np.int32)
    root = np.zeros(1, np.int32)
    lib().orc_reset_tree(children, parents, counters, root, m)
    lib().orc_build_tree(codes, children, parents, n)
    return children, parents


def compute_multipoles(px, py, pz, mass, children, parents, normalize=True):
    """tree_kernels.py:131-191 (+ :193-214 normalize_com when normalize).
    Returns (n_mass[M], n_com[M,3], n_min[M,3], n_max[M,3])."""
    px, py, pz, mass = _f32(px), _f32(py), _f32(pz), _f32(mass)
    n = px.size
    m = 2 * n - 1
    n_mass = np.zeros(m, np.float32)
    n_com = np.zeros((m, 3), np.float32)
    n_min = np.zeros((m, 3), np.float32)
    n_max = np.zeros((m, 3), np.float32)
    counts = np.zeros(m, np.int32)
    rc = lib().orc_compute_multipoles(px, py, pz, mass, np.ascontiguousarray(children),
                                      np.ascontiguousarray(parents), n_mass, n_com, n_min,
                                      n_max, counts, n)
    if rc != 0:
        raise RuntimeError("oracle: cyclic tree topology")
    if normalize:
        lib().orc_normalize_com(n_mass, n_com, m)
    return n_mass, n_com, n_min, n_max


def find_root(parents):
    """tree_kernels.py:216-234."""
    return int(lib().orc_find_root(np.ascontiguousarray(parents, np.int32), parents.size))


def build_top_tree_cache(children, root, cache_size=256):
    """tree_kernels.py:264-313 -> (top_nodes int32[cache], node_to_cache int32[M])."""
    top = np.full(cache_size, -1, np.int32)
    n2c = np.full(children.shape[0], -1, np.int32)
    lib().orc_build_top_tree_cache(np.ascontiguousarray(children, np.int32), root, top, n2c,
                                   cache_size)
    return top, n2c


def compute_forces(px, py, pz, children, n_mass, n_com, n_min, n_max, theta, G, soft, box,
                   root, off=0, count=None, nthreads=0, return_accepted=False):
    """physics_kernels.py:14-153 over targets [off, off+count).  Returns
    (force float32[N,3] with only that range written, stack_drops, visits),
    plus the number of accepted (body, node) pairs when return_accepted."""
    px, py, pz = _f32(px), _f32(py), _f32(pz)
    n = px.size
    if count is None:
        count = n - off
    force = np.zeros((n, 3), np.float32)
    visits = C.c_int64(0)
    accepted = C.c_int64(0)
    drops = lib().orc_compute_forces(px, py, pz, np.ascontiguousarray(children, np.int32),
                                     _f32(n_mass), _f32(n_com), _f32(n_min), _f32(n_max), force,
                                     theta, G, soft, box, int(root), off, count, nthreads,
                                     C.byref(visits), C.byref(accepted))
    if return_accepted:
        return force, int(drops), int(visits.value), int(accepted.value)
    return force, int(drops), int(visits.value)


def forces_targets_f64(px, py, pz, children, n_mass, n_com, n_min, n_max, theta, G, soft, box,
                       root, targets, nthreads=0):
    """physics_kernels.py:14-153 for a target list, float64 results."""
    targets = np.ascontiguousarray(targets, np.int64)
    out = np.zeros((targets.size, 3), np.float64)
    lib().orc_forces_targets_f64(_f32(px), _f32(py), _f32(pz),
                                 np.ascontiguousarray(children, np.int32), _f32(n_mass),
                                 _f32(n_com), _f32(n_min), _f32(n_max), theta, G, soft, box,
                                 int(root), targets, targets.size, out, nthreads)
    return out


def direct_sum(px, py, pz, mass, targets, G, soft, nthreads=0):
    """Float64 minimum-image direct sum for the targets (float64 [T,3])."""
    targets = np.ascontiguousarray(targets, np.int64)
    out = np.zeros((targets.size, 3), np.float64)
    px = _f32(px)
    lib().orc_direct_sum(px, _f32(py), _f32(pz), _f32(mass), px.size, targets, targets.size,
                         G, soft, out, nthreads)
    return out


def integrate(px, py, pz, vx, vy, vz, force, a, H, dt):
    """physics_kernels.py:155-203; returns updated copies (px..vz)."""
    arrs = [_f32(v).copy() for v in (px, py, pz, vx, vy, vz)]
    lib().orc_integrate(*arrs, _f32(force), arrs[0].size, a, H, dt)
    return tuple(arrs)


def render_density(px, py, pz, mvp, width, height=None):
    """render_kernels.py:12-47 on a [height, width] float32 grid.
    Returns (grid, pixel index per particle or -1)."""
    height = width if height is None else height
    px = _f32(px)
    grid = np.zeros((height, width), np.float32)
    pix = np.zeros(px.size, np.int64)
    lib().orc_render_density(px, _f32(py), _f32(pz), grid,
                             np.ascontiguousarray(mvp, np.float32).reshape(16), px.size, width,
                             height, pix.ctypes.data)
    return grid, pix


def sort_state(pos, vel, mass, key_mode):
    """src/core/state.py:20-40: codes, stable argsort, gathers."""
    codes, _ = compute_codes(*pos, key_mode=key_mode)
    perm = argsort_stable(codes)
    pos = tuple(np.ascontiguousarray(p[perm]) for p in pos)
    vel = tuple(np.ascontiguousarray(v[perm]) for v in vel)
    return pos, vel, np.ascontiguousarray(mass[perm]), codes[perm], perm


def hubble(a, H0=67.8, omega_m=1.0, omega_l=0.692):
    """src/utils/cosmology.py:76-84."""
    return H0 * np.sqrt(omega_m * a ** -3 + omega_l)


def run_reference_step(pos, vel, mass, a, da, theta, G, soft, box=1.0, key_mode=KEY_MORTON63,
                       nthreads=0):
    """One src/core/engine.py:55-123 step on the CPU.  Returns a dict with the
    sorted inputs, tree, forces and the integrated state."""
    H = hubble(a)
    dt = da / (a * H) * 0.8
    pos, vel, mass, codes, perm = sort_state(pos, vel, mass, key_mode)
    children, parents = build_tree(codes)
    n_mass, n_com, n_min, n_max = compute_multipoles(*pos, mass, children, parents)
    root = find_root(parents)
    force, drops, visits = compute_forces(*pos, children, n_mass, n_com, n_min, n_max, theta,
                                          G, soft, box, root, nthreads=nthreads)
    new = integrate(*pos, *vel, force, a, H, dt)
    return dict(pos=pos, vel=vel, mass=mass, codes=codes, perm=perm, children=children,
                parents=parents, n_mass=n_mass, n_com=n_com, n_min=n_min, n_max=n_max,
                root=root, force=force, drops=drops, visits=visits, new_pos=new[:3],
                new_vel=new[3:], a_next=a + da, H=H, dt=dt)


def colorize(grid):
    """src/utils/visualizer.py:115-171 colorize_frame in float32 numpy (the
    reference runs it in CuPy, float32).  Returns (rgb float32 [H,W,3], rgb8)."""
    g = np.asarray(grid, np.float32)
    img = np.log1p(g * np.float32(120.0))
    img = img / (img.max() + np.float32(1e-9))
    val = np.power(img, np.float32(2.2)).astype(np.float32)
    T1, T2, T3 = np.float32(0.6), np.float32(0.72), np.float32(0.82)
    r, gg, b = (np.zeros_like(val) for _ in range(3))
    m1 = val <= T1
    b[m1] = val[m1] / T1 * np.float32(0.8)
    m2 = (val > T1) & (val <= T2)
    t = (val[m2] - T1) / (T2 - T1)
    b[m2] = (1 - t) * np.float32(0.8)
    gg[m2] = t * np.float32(0.9)
    m3 = (val > T2) & (val <= T3)
    t = (val[m3] - T2) / (T3 - T2)
    gg[m3] = np.float32(0.9) + t * np.float32(0.1)
    r[m3] = t
    m4 = val > T3
    t = (val[m4] - T3) / (1 - T3)
    r[m4] = 1
    gg[m4] = 1 - t
    frame = np.clip(np.stack([r, gg, b], axis=-1) * np.float32(1.3), 0, 1).astype(np.float32)
    return frame, (frame * 255).astype(np.uint8)
