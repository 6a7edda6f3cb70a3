"""Parity at the benchmarked sizes, through the path the benchmark runs.

Integer stages (63-bit keys, the adaptive sort's permutation, children,
parents, root) and the float32 node sums, CoM, boxes of the bucketed upward
pass (unpacked to the reference layout) are compared BIT FOR BIT with the CPU
oracle on:
  * 32^3 seed 0 (one step from the initial conditions),
  * 128^3 seed 1 (the benchmark's workload), before the first step (the full
    radix sort: lattice-ordered input) and after two steps (the near-sorted
    path of the adaptive sort),
  * 128^3 seed 4 after 100 steps (the evolved state of the learned-theta
    comparison),
  * 256^3 seed 2 after 50 steps (the precision sweep's state; plus the
    topology validator).

Forces of the benchmarked traversal (grouped, the reference's opening test
decided per body: CNB_MAC_REF_X, two bodies per lane, two-level walk with
512-body super-buckets) are compared body by body with the oracle's
restatement of physics_kernels.py:14-153 in float64 at the same theta:
every body within 1e-5 of max|a| (float32 sums against float64 sums), and
the accepted (body, node) pairs counted on the device equal the oracle's
count exactly (the same node set for every body).  The bucket-decided test
(CNB_MAC_REF_X_BUCKET), which opens more nodes than the reference, is gated
on accuracy instead: its median and p99 error against the float64
minimum-image direct sum are no larger than the reference's own.
"""
import numpy as np
import pytest

from oracle import oracle as orc

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

FORCE_TOL = 1e-5       # per body, relative to max |a| of the sample


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _cfg(n_grid, **kw):
    from cnb.utils import config as cfgmod
    base = dict(N_GRID=n_grid, SOFTENING=0.5 / n_grid, THETA=0.5, KEY_MODE="morton63",
                FORCE_MODE="grouped", MAC="ref_x", BODIES_PER_LANE=2, BLOCK_WARPS=2,
                SUPER_BODIES=512, N_STEPS=1000, A_START=0.02, A_END=0.02 + 1000 * 0.002)
    base.update(kw)
    return cfgmod.make(**base)


def _engine(n_grid, seed, steps=0, **kw):
    from cnb.core.engine import SimulationEngine
    from cnb.core.state import SimulationState
    from cnb.utils.cosmology import zeldovich_tensors
    pos, vel = zeldovich_tensors(n_grid, seed, "cuda")
    eng = SimulationEngine(_cfg(n_grid, **kw), SimulationState(n_grid ** 3, pos, vel), camera=False)
    for _ in range(steps):
        eng.step()
    eng.check()
    return eng


def _host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def _integer_stages(eng):
    """Sort and tree of the engine's current state against the oracle, bit for
    bit; returns the oracle's sorted positions, masses, tree and root."""
    s, tm = eng.state, eng.tree_manager
    pos_h = [_host(p) for p in s.pos]
    s.sort_buffer_by_morton(eng.config)
    tm.build(s.pos, s.mass, s.codes)
    eng.check()
    want_codes, _ = orc.compute_codes(*pos_h, orc.KEY_MORTON63)
    want_perm = np.argsort(want_codes, kind="stable")
    np.testing.assert_array_equal(_host(s.perm).astype(np.int64), want_perm)
    codes = want_codes[want_perm]
    np.testing.assert_array_equal(_host(s.codes), codes)
    spos = [np.ascontiguousarray(p[want_perm]) for p in pos_h]
    for got, want in zip(s.pos, spos):
        np.testing.assert_array_equal(_host(got), want)
    ch, par = orc.build_tree(codes)
    buf = tm.get_buffers()
    np.testing.assert_array_equal(_host(buf["child"]), ch)
    np.testing.assert_array_equal(_host(tm.parent), par)
    assert int(_host(buf["root"])[0]) == orc.find_root(par)
    mass = _host(s.mass)
    wm, wc, wlo, whi = orc.compute_multipoles(*spos, mass, ch, par)
    for key, want in (("mass", wm), ("com", wc), ("min", wlo), ("max", whi)):
        np.testing.assert_array_equal(_host(buf[key]).view(np.uint32), want.view(np.uint32), err_msg=key)
    return spos, mass, (ch, wm, wc, wlo, whi), orc.find_root(par)


def _forces_vs_reference(eng, spos, tree, root, targets, theta=0.5):
    """Device forces of the engine's traversal on the current (sorted) state
    and the oracle's float64 traversal at the same theta, for the targets."""
    ch, wm, wc, wlo, whi = tree
    eng.stats.zero_()
    eng.compute_forces()
    eng.check()
    got = _host(eng.state.force)[targets].astype(np.float64)
    soft = float(eng.config.SOFTENING)
    want = orc.forces_targets_f64(*spos, ch, wm, wc, wlo, whi, theta, 1.0, soft, 1.0, root, targets)
    return got, want


def _check_same_forces(got, want):
    amax = np.abs(want).max()
    err = np.linalg.norm(got - want, axis=1)
    worst = float(err.max() / amax)
    assert worst <= FORCE_TOL, f"worst body {worst:.3g} of max|a|"
    return worst


def _sample(n, seed=0, k=4096):
    return np.sort(np.random.default_rng(seed).choice(n, min(k, n), replace=False)).astype(np.int64)


@pytest.mark.parametrize("bpl,warps,super_bodies", [(2, 2, 512), (2, 4, 0), (1, 8, 0), (1, 4, 1024)])
def test_cfg1_every_body_gets_the_reference_nodes(bpl, warps, super_bodies):
    """32^3 seed 0: every body's force equals the reference traversal's and the
    accepted (body, node) pairs are exactly the oracle's."""
    eng = _engine(32, 0, BODIES_PER_LANE=bpl, BLOCK_WARPS=warps, SUPER_BODIES=super_bodies)
    spos, _, tree, root = _integer_stages(eng)
    ch, wm, wc, wlo, whi = tree
    eng.stats.zero_()
    eng.compute_forces()
    eng.check()
    got = _host(eng.state.force).astype(np.float64)
    want, drops, _, accepted = orc.compute_forces(*spos, ch, wm, wc, wlo, whi, 0.5, 1.0, 0.5 / 32, 1.0,
                                                  root, return_accepted=True)
    assert drops == 0
    _check_same_forces(got, want.astype(np.float64))
    assert int(_host(eng.stats)[0]) == accepted


@pytest.mark.parametrize("theta", [0.3, 0.7, 1.0])
def test_cfg1_other_angles(theta):
    eng = _engine(32, 0, THETA=theta)
    spos, _, tree, root = _integer_stages(eng)
    ch, wm, wc, wlo, whi = tree
    eng.stats.zero_()
    eng.compute_forces()
    eng.check()
    want, _, _, accepted = orc.compute_forces(*spos, ch, wm, wc, wlo, whi, theta, 1.0, 0.5 / 32, 1.0,
                                              root, return_accepted=True)
    _check_same_forces(_host(eng.state.force).astype(np.float64), want.astype(np.float64))
    assert int(_host(eng.stats)[0]) == accepted


def test_cfg2_benchmark_workload():
    """128^3 seed 1: integer stages bit-exact on the full sort (first step) and
    on the near-sorted path (after two steps), forces of the benchmarked
    traversal equal to the reference's on a 4 096-body sample."""
    eng = _engine(128, 1)
    spos, _, tree, root = _integer_stages(eng)          # lattice order: full radix sort
    near0, _ = eng.state._ctx.stats()
    t = _sample(eng.state.n)
    got, want = _forces_vs_reference(eng, spos, tree, root, t)
    worst = _check_same_forces(got, want)
    print(f"128^3 seed 1, step 0: worst body {worst:.2e} of max|a|")
    for _ in range(2):
        eng.step()
    eng.check()
    spos, _, tree, root = _integer_stages(eng)          # sorted one step earlier: near-sorted path
    near1, _ = eng.state._ctx.stats()
    assert near1 > near0, "the near-sorted path was not taken"
    got, want = _forces_vs_reference(eng, spos, tree, root, t)
    _check_same_forces(got, want)


def test_cfg5_evolved_state():
    """128^3 seed 4 after 100 steps: integer stages and forces."""
    eng = _engine(128, 4, steps=100)
    spos, _, tree, root = _integer_stages(eng)
    got, want = _forces_vs_reference(eng, spos, tree, root, _sample(eng.state.n, 4))
    _check_same_forces(got, want)


def test_cfg3_256cube_after_50_steps():
    """256^3 seed 2 after 50 steps: keys, permutation, topology and node sums
    bit-exact, the topology validator clean, forces on a sample."""
    eng = _engine(256, 2, steps=50)
    spos, _, tree, root = _integer_stages(eng)
    eng.tree_manager.validate()
    got, want = _forces_vs_reference(eng, spos, tree, root, _sample(eng.state.n, 2, 1024))
    _check_same_forces(got, want)


def test_bucket_test_is_at_least_as_accurate():
    """CNB_MAC_REF_X_BUCKET opens every node that some body of the bucket
    would open: not the reference's node sets, but its error against the
    float64 direct sum is no larger than the reference's (median and p99 of
    |a - a_direct| / |a_direct| on a 4 096-body sample of 128^3 seed 1)."""
    from cnb import _lib
    eng = _engine(128, 1, MAC="ref_x_bucket")
    spos, _, tree, root = _integer_stages(eng)
    t = _sample(eng.state.n)
    eng.compute_forces()
    eng.check()
    got = _host(eng.state.force)[t].astype(np.float64)
    ch, wm, wc, wlo, whi = tree
    ref = orc.forces_targets_f64(*spos, ch, wm, wc, wlo, whi, 0.5, 1.0, 0.5 / 128, 1.0, root, t)
    T = torch.from_numpy(t).cuda()
    out = torch.empty((t.size, 3), dtype=torch.float64, device="cuda")
    _lib.call("cnb_direct_sum_f64", *(p.data_ptr() for p in eng.state.pos), eng.state.mass.data_ptr(),
              eng.state.n, T.data_ptr(), t.size, 1.0, 0.5 / 128, out.data_ptr(),
              int(torch.cuda.current_stream().cuda_stream))
    d = _host(out)
    nd = np.linalg.norm(d, axis=1)
    e_bucket = np.linalg.norm(got - d, axis=1) / nd
    e_ref = np.linalg.norm(ref - d, axis=1) / nd
    print(f"bucket test: median {np.median(e_bucket):.3g} p99 {np.percentile(e_bucket, 99):.3g}; "
          f"reference: median {np.median(e_ref):.3g} p99 {np.percentile(e_ref, 99):.3g}")
    assert np.median(e_bucket) <= np.median(e_ref)
    assert np.percentile(e_bucket, 99) <= np.percentile(e_ref, 99)
