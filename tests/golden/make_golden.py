"""Generate the golden fixtures in tests/golden/ from the reference itself.

Runs Cosmo-NBody's own kernels (src/kernels/*.py, read from the reference
checkout given by --ref) under Numba's CUDA simulator
(NUMBA_ENABLE_CUDASIM=1; no GPU needed) on small seeded Zel'dovich inputs and
stores inputs and outputs as .npz.  Only the reference's kernels are
executed; `cp.argsort` (src/core/state.py:35) is replaced by a stable numpy
argsort and the gathers by numpy indexing.  The reference's modules import
cupy without using it on these paths; a stub module stands in for it.

The simulator evaluates float arithmetic with NumPy promotion rules
(float32 stays float32) where compiled Numba promotes to float64, so the
float outputs here pin the oracle to a tolerance, the integer outputs
(keys, order, topology) and the float32 sums/min/max exactly.

    python tests/golden/make_golden.py --ref /root/reference
"""
from __future__ import annotations

import argparse
import os
import sys
import time
import types

os.environ["NUMBA_ENABLE_CUDASIM"] = "1"
import numpy as np  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "cosmo-nbody_b200"))


def _cupy_stub():
    cp = types.ModuleType("cupy")
    cp.asarray = np.asarray
    cp.float32 = np.float32
    cp.int32 = np.int32
    sys.modules["cupy"] = cp


def _morton63(x, y, z):
    def s(v):
        r = np.zeros_like(v)
        for b in range(21):
            r |= ((v >> np.uint64(b)) & np.uint64(1)) << np.uint64(3 * b)
        return r
    lim = np.uint64((1 << 21) - 1)
    ix = np.minimum((x.astype(np.float64) * 2097152.0).astype(np.uint64), lim)
    iy = np.minimum((y.astype(np.float64) * 2097152.0).astype(np.uint64), lim)
    iz = np.minimum((z.astype(np.float64) * 2097152.0).astype(np.uint64), lim)
    return s(ix) | (s(iy) << np.uint64(1)) | (s(iz) << np.uint64(2))


def run_case(ref, n_grid, seed, key_mode, force_targets, theta=0.5):
    from cnb.utils.cosmology import zeldovich_arrays
    from src.kernels.morton import compute_codes
    from src.kernels.tree_kernels import (build_tree, build_top_tree_cache, compute_multipoles,
                                          find_root, normalize_com, reset_tree_buffers)
    from src.kernels.physics_kernels import compute_forces, integrate
    from src.kernels.render_kernels import render_density
    from src.utils import config as rcfg
    from src.utils.visualizer import get_mvp_matrix

    pos, vel = zeldovich_arrays(n_grid, seed)
    n = n_grid ** 3
    m = 2 * n - 1
    tpb = 256
    bpg = (n + tpb - 1) // tpb
    x, y, z = [p.copy() for p in pos]
    out = {"n_grid": n_grid, "seed": seed, "theta": theta, "px0": x, "py0": y, "pz0": z,
           "vx0": vel[0], "vy0": vel[1], "vz0": vel[2]}

    codes = np.zeros(n, np.uint64)
    indices = np.zeros(n, np.uint32)
    compute_codes[bpg, tpb](x, y, z, codes, indices, n)
    out["codes_compat30"] = codes.copy()
    out["indices"] = indices.copy()
    keys = codes if key_mode == "compat30" else _morton63(x, y, z)
    perm = np.argsort(keys, kind="stable")
    out["perm"] = perm.astype(np.int64)
    sx, sy, sz = x[perm], y[perm], z[perm]
    skeys = np.ascontiguousarray(keys[perm])
    mass = np.full(n, 1.0 / n, np.float32)
    out["mass"] = mass

    child = np.full((m, 2), -1, np.int32)
    parent = np.full(m, -1, np.int32)
    counters = np.zeros(m, np.int32)
    root = np.zeros(1, np.int32)
    reset_tree_buffers[(m + tpb - 1) // tpb, tpb](child, parent, counters, root)
    build_tree[bpg, tpb](skeys, child, parent)
    out["children"] = child.copy()
    out["parents"] = parent.copy()

    n_mass = np.zeros(m, np.float32)
    n_com = np.zeros((m, 3), np.float32)
    n_min = np.zeros((m, 3), np.float32)
    n_max = np.zeros((m, 3), np.float32)
    compute_multipoles[bpg, tpb](sx, sy, sz, mass, child, parent, n_mass, n_com, n_min, n_max,
                                 counters)
    out["n_mass"] = n_mass.copy()
    out["n_com_raw"] = n_com.copy()
    out["n_min"] = n_min.copy()
    out["n_max"] = n_max.copy()
    normalize_com[(m + 255) // 256, 256](n_mass, n_com, m)
    out["n_com"] = n_com.copy()
    find_root[(m + tpb - 1) // tpb, tpb](parent, root)
    out["root"] = root.copy()
    top = np.full(256, -1, np.int32)
    n2c = np.full(m, -1, np.int32)
    build_top_tree_cache[1, 1](child, root, top, n2c, 256)
    out["top_nodes"] = top.copy()
    out["node_to_cache"] = n2c.copy()

    soft = 0.5 / n_grid
    force = np.zeros((n, 3), np.float32)
    targets = []
    for off in force_targets:
        compute_forces[1, tpb](sx, sy, sz, child, n_mass, n_com, n_min, n_max, force, theta, 1.0,
                               soft, 1.0, root, top, n2c, off)
        targets.append(np.arange(off, min(off + tpb, n)))
    t = np.concatenate(targets)
    out["force_targets"] = t
    out["force"] = force[t].copy()
    out["soft"] = soft

    a, H, dt = 0.02, 67.8 * np.sqrt(1.0 * 0.02 ** -3 + 0.692), 1e-4
    ix, iy, iz = sx.copy(), sy.copy(), sz.copy()
    ivx, ivy, ivz = vel[0][perm].copy(), vel[1][perm].copy(), vel[2][perm].copy()
    fint = np.zeros((n, 3), np.float32)
    fint[t] = force[t]
    integrate[bpg, tpb](ix, iy, iz, ivx, ivy, ivz, fint, a, H, dt)
    out.update(int_a=a, int_H=H, int_dt=dt, int_px=ix, int_py=iy, int_pz=iz, int_vx=ivx,
               int_vy=ivy, int_vz=ivz)

    res = 128
    grid = np.zeros((res, res), np.float32)
    mvp = np.asarray(get_mvp_matrix(3, (0.5, 0.5, 0.5), 1.0, rcfg), np.float32)
    render_density[bpg, tpb](sx, sy, sz, grid, mvp, res)
    out["mvp"] = mvp
    out["grid"] = grid
    out["key_mode"] = key_mode
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    args = ap.parse_args()
    _cupy_stub()
    sys.path.insert(0, args.ref)
    cases = [
        (8, 0, "compat30", [0, 256]),
        (8, 0, "morton63", [0, 256]),
        (16, 0, "compat30", [0, 2048]),
        (16, 0, "morton63", [0, 2048]),
    ]
    for n_grid, seed, key_mode, ft in cases:
        t0 = time.time()
        out = run_case(args.ref, n_grid, seed, key_mode, ft)
        name = os.path.join(HERE, f"ref_n{n_grid}_s{seed}_{key_mode}.npz")
        np.savez_compressed(name, **out)
        print(f"{name}: {time.time() - t0:.1f} s", flush=True)


if __name__ == "__main__":
    main()
