"""Pins the CPU oracle against the reference's own kernels.

The fixtures in tests/golden/ were produced by running Cosmo-NBody's kernels
(src/kernels/*.py) under Numba's CUDA simulator (tests/golden/make_golden.py).
Integer stages and float32 sums / min / max must match bit for bit; stages
whose float arithmetic the simulator evaluates in float32 (compiled Numba:
float64) match to a stated tolerance.
"""
import numpy as np
import pytest

from oracle import oracle as orc


def _load(path):
    d = np.load(path, allow_pickle=False)
    return {k: d[k] for k in d.files}


def _mode(g):
    return orc.KEY_COMPAT30 if str(g["key_mode"]) == "compat30" else orc.KEY_MORTON63


def test_fixtures_present(golden_files):
    assert len(golden_files) >= 4


def test_keys_bit_exact(golden_files):
    for f in golden_files:
        g = _load(f)
        codes, idx = orc.compute_codes(g["px0"], g["py0"], g["pz0"], orc.KEY_COMPAT30)
        np.testing.assert_array_equal(codes, g["codes_compat30"], err_msg=f)
        np.testing.assert_array_equal(idx, g["indices"], err_msg=f)
        # the reference's key is a 30-bit key of the low 10 bits of each coordinate
        assert int(codes.max()) < (1 << 30)


def test_sort_order_bit_exact(golden_files):
    for f in golden_files:
        g = _load(f)
        codes, _ = orc.compute_codes(g["px0"], g["py0"], g["pz0"], _mode(g))
        np.testing.assert_array_equal(orc.argsort_stable(codes), g["perm"], err_msg=f)


def test_topology_bit_exact(golden_files):
    for f in golden_files:
        g = _load(f)
        codes, _ = orc.compute_codes(g["px0"], g["py0"], g["pz0"], _mode(g))
        perm = orc.argsort_stable(codes)
        ch, par = orc.build_tree(codes[perm])
        np.testing.assert_array_equal(ch, g["children"], err_msg=f)
        np.testing.assert_array_equal(par, g["parents"], err_msg=f)
        assert orc.find_root(par) == int(g["root"][0])


def _tree(g):
    codes, _ = orc.compute_codes(g["px0"], g["py0"], g["pz0"], _mode(g))
    perm = orc.argsort_stable(codes)
    pos = [g[k][perm] for k in ("px0", "py0", "pz0")]
    ch, par = orc.build_tree(codes[perm])
    return pos, ch, par


def test_multipoles_bit_exact(golden_files):
    for f in golden_files:
        g = _load(f)
        pos, ch, par = _tree(g)
        m, c, lo, hi = orc.compute_multipoles(*pos, g["mass"], ch, par, normalize=False)
        np.testing.assert_array_equal(m, g["n_mass"], err_msg=f)
        np.testing.assert_array_equal(c, g["n_com_raw"], err_msg=f)
        np.testing.assert_array_equal(lo, g["n_min"], err_msg=f)
        np.testing.assert_array_equal(hi, g["n_max"], err_msg=f)


def test_normalized_com_within_one_ulp(golden_files):
    # the simulator computes 1.0 / m in float32; compiled Numba (and the
    # oracle) in float64, so the stored float32 CoM may differ by one ulp
    for f in golden_files:
        g = _load(f)
        pos, ch, par = _tree(g)
        _, c, _, _ = orc.compute_multipoles(*pos, g["mass"], ch, par, normalize=True)
        ulp = np.spacing(np.abs(g["n_com"]).astype(np.float32))
        assert np.all(np.abs(c - g["n_com"]) <= 2 * ulp), f


def test_top_tree_cache_bit_exact(golden_files):
    for f in golden_files:
        g = _load(f)
        _, ch, par = _tree(g)
        top, n2c = orc.build_top_tree_cache(ch, orc.find_root(par), 256)
        np.testing.assert_array_equal(top, g["top_nodes"], err_msg=f)
        np.testing.assert_array_equal(n2c, g["node_to_cache"], err_msg=f)


def test_forces_match_reference(golden_files):
    # float32 (simulator) vs float64 (oracle) arithmetic: relative to the
    # largest acceleration of the sample
    for f in golden_files:
        g = _load(f)
        pos, ch, par = _tree(g)
        m, c, lo, hi = orc.compute_multipoles(*pos, g["mass"], ch, par)
        t = g["force_targets"]
        out = orc.forces_targets_f64(*pos, ch, m, c, lo, hi, float(g["theta"]), 1.0,
                                     float(g["soft"]), 1.0, orc.find_root(par), t)
        scale = np.abs(out).max()
        err = np.abs(out - g["force"]).max() / scale
        assert err < 2e-4, (f, err)


def test_integrate_matches_reference(golden_files):
    for f in golden_files:
        g = _load(f)
        pos, _, _ = _tree(g)
        perm = g["perm"]
        vel = [g[k][perm] for k in ("vx0", "vy0", "vz0")]
        t = g["force_targets"]
        force = np.zeros((pos[0].size, 3), np.float32)
        force[t] = g["force"]
        new = orc.integrate(*pos, *vel, force, float(g["int_a"]), float(g["int_H"]),
                            float(g["int_dt"]))
        for k, key in enumerate(("int_px", "int_py", "int_pz", "int_vx", "int_vy", "int_vz")):
            ref = g[key]
            tol = 4 * np.spacing(np.maximum(np.abs(ref), 1e-30).astype(np.float32))
            bad = np.abs(new[k] - ref) > tol
            # float32 (simulator) vs float64 rounding of the kick; wrap-around
            # across 1.0 may differ by exactly one period
            wrap = np.abs(np.abs(new[k] - ref) - 1.0) < 1e-6
            assert np.all(~bad | wrap), (f, key, np.abs(new[k] - ref).max())


def test_render_matches_reference(golden_files):
    for f in golden_files:
        g = _load(f)
        pos, _, _ = _tree(g)
        res = g["grid"].shape[0]
        grid, pix = orc.render_density(*pos, g["mvp"], res)
        ref = g["grid"]
        assert abs(grid.sum() - ref.sum()) <= 1e-5 * ref.sum(), f
        # per-pixel: identical up to float32 summation order / rounding
        np.testing.assert_allclose(grid, ref, rtol=1e-5, atol=1e-4 * ref.max(), err_msg=f)


def test_direct_sum_antisymmetry():
    rng = np.random.default_rng(3)
    n = 64
    x, y, z = (rng.random(n).astype(np.float32) for _ in range(3))
    mass = np.full(n, 1.0 / n, np.float32)
    acc = orc.direct_sum(x, y, z, mass, np.arange(n), 1.0, 0.01)
    # equal masses: total momentum change is zero (pairwise antisymmetric law)
    assert np.abs(acc.sum(axis=0)).max() < 1e-9 * np.abs(acc).max()



def test_mvp_matches_reference(golden_files):
    """cnb.utils.visualizer.get_mvp_matrix at the reference's square aspect
    equals the matrix the reference's own get_mvp_matrix produced
    (src/utils/visualizer.py:81-112, recorded in each fixture by
    make_golden.py for step 3, centre (0.5, 0.5, 0.5), box 1)."""
    from cnb.utils import config as cfgmod
    from cnb.utils.visualizer import get_mvp_matrix
    got = get_mvp_matrix(3, (0.5, 0.5, 0.5), 1.0, cfgmod.make())
    assert got.dtype == np.float32
    for f in golden_files:
        np.testing.assert_array_equal(got, _load(f)["mvp"])
