"""Two-level grouped traversal (cnb_forces_two_level): super-buckets walk the
top of the tree once for all their buckets.  It accepts the same nodes as the
single-level traversal with the same form of the reference's opening test
(per body, CNB_MAC_REF_X = 0, or per bucket, CNB_MAC_REF_X_BUCKET = 3), so its forces equal
cnb_forces_grouped's up to float32 summation order and its interaction count
is the same; at theta = 0 it is the minimum-image direct sum.  Super-buckets
whose lists do not fit fall back to the walk from the root."""
import numpy as np
import pytest

from oracle import oracle as orc

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _bodies(kind, n_grid, seed):
    from cnb.utils.cosmology import zeldovich_arrays
    if kind == "zeldovich":
        (x, y, z), _ = zeldovich_arrays(n_grid, seed)
    elif kind == "clustered":
        # a few tight clumps plus a uniform background
        rng = np.random.default_rng(seed)
        n = n_grid ** 3
        centres = rng.random((8, 3))
        k = rng.integers(0, 8, n)
        p = centres[k] + rng.normal(0, 0.01, (n, 3))
        bg = rng.random(n) < 0.3
        p[bg] = rng.random((int(bg.sum()), 3))
        x, y, z = (np.mod(p[:, i], 1.0).astype(np.float32) for i in range(3))
    elif kind == "close_pairs":
        # companions planted next to 90 bodies at distances on both sides of
        # the reference's cut d^2 > 1e-7 (sqrt = 3.16e-4), one coincident
        (x, y, z), _ = zeldovich_arrays(n_grid, seed)
        x, y, z = (np.array(a, np.float64) for a in (x, y, z))
        rng = np.random.default_rng(seed + 7)
        n = x.size
        idx = rng.choice(np.arange(0, n - 1, 2), 90, replace=False)
        dist = np.array([0.0, 1e-4, 2.5e-4, 3.0e-4, 3.4e-4, 4e-4, 1e-3])
        for k, i in enumerate(idx):
            u = rng.normal(size=3)
            u /= np.linalg.norm(u)
            d = dist[k % dist.size] * u
            x[i + 1], y[i + 1], z[i + 1] = x[i] + d[0], y[i] + d[1], z[i] + d[2]
        x, y, z = (np.mod(a, 1.0).astype(np.float32) for a in (x, y, z))
    else:
        raise ValueError(kind)
    codes, _ = orc.compute_codes(x, y, z, 1)
    perm = orc.argsort_stable(codes)
    return [a[perm] for a in (x, y, z)], codes[perm]


class Case:
    def __init__(self, kind, n_grid, seed=0, bpl=1, soft=None, mac=0):
        from cnb.core.octree import OctreeManager
        pos, codes = _bodies(kind, n_grid, seed)
        self.pos_h = pos
        self.n = n = codes.size
        self.P = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in pos]
        self.M = torch.full((n,), 1.0 / n, device="cuda")
        self.bpl = bpl
        self.tm = OctreeManager(n, node_table=True, bucket=32 * bpl)
        self.tm.build(self.P, self.M, torch.from_numpy(codes).cuda())
        self.soft = 0.5 / n_grid if soft is None else soft
        self.st = int(torch.cuda.current_stream().cuda_stream)
        self.mac = mac

    def single(self, theta, warps=4):
        from cnb import _lib
        f = torch.empty((self.n, 3), device="cuda")
        stats = torch.zeros(4, dtype=torch.int64, device="cuda")
        status = torch.zeros(1, dtype=torch.int32, device="cuda")
        _lib.call("cnb_forces_grouped", *(p.data_ptr() for p in self.P), self.tm.node_table.data_ptr(),
                  self.tm.workspace.data_ptr(), f.data_ptr(), self.n, theta, None, self.mac,
                  self.bpl, warps, 1.0, self.soft, 1.0, 0.0, stats.data_ptr(), status.data_ptr(), self.st)
        torch.cuda.synchronize()
        assert int(status.item()) == 0
        return f.cpu().numpy(), stats.cpu().numpy()

    def two_level(self, theta, super_bodies, warps=4, ws_bytes=None):
        from cnb import _lib
        nbytes = _lib.load().cnb_two_level_workspace_bytes(self.n, super_bodies)
        if ws_bytes is not None:
            nbytes = ws_bytes
        ws = torch.zeros((nbytes + 15) // 16 * 4, dtype=torch.int32, device="cuda")
        f = torch.empty((self.n, 3), device="cuda")
        stats = torch.zeros(4, dtype=torch.int64, device="cuda")
        status = torch.zeros(1, dtype=torch.int32, device="cuda")
        _lib.call("cnb_forces_two_level", *(p.data_ptr() for p in self.P), self.tm.node_table.data_ptr(),
                  self.tm.ranges.data_ptr(), self.tm.parent.data_ptr(), self.tm.workspace.data_ptr(),
                  ws.data_ptr(), nbytes, super_bodies, f.data_ptr(), self.n, theta, self.mac, self.bpl, warps,
                  1.0, self.soft, 1.0, stats.data_ptr(), status.data_ptr(), self.st)
        torch.cuda.synchronize()
        assert int(status.item()) == 0
        hdr = ws.cpu().numpy()
        return f.cpu().numpy(), stats.cpu().numpy(), hdr[:4]


def _close(f2, f1, rel=2e-4):
    rms = np.sqrt(np.mean(np.sum(f1.astype(np.float64) ** 2, axis=1)))
    err = np.linalg.norm(f2.astype(np.float64) - f1, axis=1)
    assert np.isfinite(f2).all()
    assert err.max() <= rel * rms, (err.max() / rms)


@pytest.mark.parametrize("mac", [0, 3])
@pytest.mark.parametrize("kind,n_grid,bpl,super_bodies", [
    ("zeldovich", 32, 1, 1024), ("zeldovich", 32, 2, 512), ("clustered", 32, 1, 256),
    ("clustered", 24, 2, 2048), ("zeldovich", 16, 1, 64)])
def test_same_nodes_as_single_level(kind, n_grid, bpl, super_bodies, mac):
    c = Case(kind, n_grid, 1, bpl, mac=mac)
    f1, s1 = c.single(0.5)
    f2, s2, hdr = c.two_level(0.5, super_bodies)
    _close(f2, f1)
    # the same accepted nodes: equal body-node interaction counts
    assert abs(int(s2[0]) - int(s1[0])) <= 1e-4 * int(s1[0])
    assert int(hdr[0]) > 0          # super-buckets were built
    assert int(hdr[2]) < int(hdr[0])  # and most of them fit their lists


@pytest.mark.parametrize("mac", [0, 3])
@pytest.mark.parametrize("theta", [0.3, 0.7, 1.0])
def test_theta_range(theta, mac):
    c = Case("zeldovich", 24, 2, mac=mac)
    f1, s1 = c.single(theta)
    f2, s2, _ = c.two_level(theta, 1024)
    _close(f2, f1)
    assert abs(int(s2[0]) - int(s1[0])) <= 1e-4 * int(s1[0])


def test_theta_zero_is_direct_sum():
    # every leaf lands in the super-buckets' far lists (512 bodies fit)
    c = Case("zeldovich", 8, 3)
    f2, s2, hdr = c.two_level(0.0, 64)
    assert int(hdr[2]) == 0
    assert int(s2[0]) == c.n * c.n
    d = orc.direct_sum(*c.pos_h, np.full(c.n, 1.0 / c.n, np.float32), np.arange(c.n), 1.0, c.soft)
    _close(f2, d, 1e-4)


@pytest.mark.parametrize("mac", [0, 3])
@pytest.mark.parametrize("bpl", [1, 2])
def test_cut_close_pairs(bpl, mac):
    """The reference's cut (no force from a node at d^2 <= 1e-7): with a small
    softening the planted pairs inside the cut would dominate the force if
    they were applied, and those just outside it must be.  Both traversals at
    theta -> 0 (every entry a leaf) are the direct sum with the cut; at
    theta = 0.5 they accept the same nodes and agree."""
    c = Case("close_pairs", 16, 2, bpl, soft=1e-4, mac=mac)
    m = np.full(c.n, 1.0 / c.n, np.float32)
    d = orc.direct_sum(*c.pos_h, m, np.arange(c.n), 1.0, c.soft)
    f1, _ = c.single(1e-6)
    f2, _, hdr = c.two_level(1e-6, 64)
    _close(f1, d, 1e-4)
    _close(f2, d, 1e-4)
    f1, _ = c.single(0.5)
    f2, _, _ = c.two_level(0.5, 512)
    _close(f2, f1)


def test_overflowing_lists_fall_back_to_root_walk():
    # theta = 0 with 4096 bodies overflows every far list: all super-buckets
    # are incomplete and every bucket walks from the root
    c = Case("zeldovich", 16, 4)
    f1, s1 = c.single(0.0)
    f2, s2, hdr = c.two_level(0.0, 256)
    assert int(hdr[2]) == int(hdr[0])
    _close(f2, f1, 1e-5)
    assert int(s2[0]) == int(s1[0]) == c.n * c.n


def test_small_workspace_lists_few_super_buckets():
    from cnb import _lib
    c = Case("zeldovich", 16, 5)
    f1, s1 = c.single(0.5)
    # the layout: 16-byte header, n super-bucket records, n body slots, then list slots
    fixed = 16 + 16 * c.n + (4 * c.n + 15) // 16 * 16
    slot = 16 + 4 * 256 + 16 * 2048
    assert _lib.load().cnb_two_level_workspace_bytes(c.n, 64) >= fixed + slot
    f2, s2, hdr = c.two_level(0.5, 64, ws_bytes=fixed + 3 * slot)
    assert int(hdr[0]) > 3
    _close(f2, f1)
    assert abs(int(s2[0]) - int(s1[0])) <= 1e-4 * int(s1[0])
    # below one list slot the call is rejected before any launch
    with pytest.raises(_lib.CnbError):
        c.two_level(0.5, 64, ws_bytes=fixed + slot - 16)


@pytest.mark.parametrize("n", [1, 2, 3, 33, 100])
def test_tiny_systems(n):
    from cnb import _lib
    from cnb.core.octree import OctreeManager
    rng = np.random.default_rng(n)
    p = rng.random((n, 3)).astype(np.float32)
    codes, _ = orc.compute_codes(p[:, 0], p[:, 1], p[:, 2], 1)
    perm = orc.argsort_stable(codes)
    p, codes = p[perm], codes[perm]
    P = [torch.from_numpy(np.ascontiguousarray(p[:, i])).cuda() for i in range(3)]
    M = torch.full((n,), 1.0 / n, device="cuda")
    tm = OctreeManager(n, node_table=True)
    tm.build(P, M, torch.from_numpy(codes).cuda())
    st = int(torch.cuda.current_stream().cuda_stream)
    out = {}
    for theta in (0.0, 0.5):
        nbytes = _lib.load().cnb_two_level_workspace_bytes(n, 32)
        ws = torch.zeros((nbytes + 15) // 16 * 4, dtype=torch.int32, device="cuda")
        f2 = torch.empty((n, 3), device="cuda")
        f1 = torch.empty((n, 3), device="cuda")
        status = torch.zeros(1, dtype=torch.int32, device="cuda")
        _lib.call("cnb_forces_two_level", *(q.data_ptr() for q in P), tm.node_table.data_ptr(),
                  tm.ranges.data_ptr(), tm.parent.data_ptr(), tm.workspace.data_ptr(), ws.data_ptr(),
                  nbytes, 32, f2.data_ptr(), n, theta, _lib.MAC_REF_X, 1, 4, 1.0, 0.01, 1.0, None,
                  status.data_ptr(), st)
        _lib.call("cnb_forces_grouped", *(q.data_ptr() for q in P), tm.node_table.data_ptr(),
                  tm.workspace.data_ptr(), f1.data_ptr(), n, theta, None, _lib.MAC_REF_X, 1, 4, 1.0,
                  0.01, 1.0, 0.0, None, status.data_ptr(), st)
        torch.cuda.synchronize()
        assert int(status.item()) == 0
        out[theta] = f2.cpu().numpy(), f1.cpu().numpy()
    f2, f1 = out[0.5]
    np.testing.assert_allclose(f2, f1, rtol=1e-4, atol=1e-6)
    # theta = 0: the minimum-image direct sum
    d = orc.direct_sum(p[:, 0], p[:, 1], p[:, 2], np.full(n, 1.0 / n, np.float32), np.arange(n), 1.0, 0.01)
    np.testing.assert_allclose(out[0.0][0], d, rtol=1e-4, atol=1e-6)


def test_engine_two_level_matches_single_level():
    from cnb.core.engine import SimulationEngine
    from cnb.core.state import SimulationState
    from cnb.utils import config as cfgmod
    from cnb.utils.cosmology import zeldovich_arrays
    forces = []
    for sb in (0, 1024):
        cfg = cfgmod.make(N_GRID=24, SOFTENING=0.5 / 24, THETA=0.5, N_STEPS=100, A_START=0.02,
                          A_END=0.22, KEY_MODE="morton63", FORCE_MODE="grouped", BODIES_PER_LANE=2,
                          BLOCK_WARPS=4, SUPER_BODIES=sb)
        pos, vel = zeldovich_arrays(24, 2)
        st = SimulationState(24 ** 3, pos, vel)
        eng = SimulationEngine(cfg, st, camera=False)
        eng.forces_only()
        eng.check()
        forces.append(st.force.cpu().numpy())
    _close(forces[1], forces[0])


def test_super_size_change_between_builds():
    """The tree build makes the super-bucket table for the engine's current
    super-bucket size; after a change of size (as the autotuner makes) the
    next force call, before any rebuild, makes the table itself and gives the
    same forces as the single-level walk."""
    from cnb.core.engine import SimulationEngine
    from cnb.core.state import SimulationState
    from cnb.utils import config as cfgmod
    from cnb.utils.cosmology import zeldovich_arrays
    cfg = cfgmod.make(N_GRID=24, SOFTENING=0.5 / 24, THETA=0.5, N_STEPS=100, A_START=0.02,
                      A_END=0.22, KEY_MODE="morton63", FORCE_MODE="grouped", BODIES_PER_LANE=2,
                      BLOCK_WARPS=4, SUPER_BODIES=512)
    pos, vel = zeldovich_arrays(24, 3)
    st = SimulationState(24 ** 3, pos, vel)
    eng = SimulationEngine(cfg, st, camera=False)
    eng.forces_only()
    eng.check()
    tm = eng.tree_manager
    assert tm.super_table_current
    f512 = st.force.clone()
    eng.set_super_bodies(1024)
    assert not tm.super_table_current
    st.force.zero_()
    eng.compute_forces()
    eng.check()
    f1024 = st.force.clone()
    eng.set_super_bodies(0)
    st.force.zero_()
    eng.compute_forces()
    eng.check()
    f0 = st.force.cpu().numpy()
    _close(f512.cpu().numpy(), f0)
    _close(f1024.cpu().numpy(), f0)
    # the next build makes the 1024-body table again
    eng.set_super_bodies(1024)
    eng.forces_only()
    eng.check()
    assert tm.super_table_current
    _close(st.force.cpu().numpy(), f0)


@pytest.mark.parametrize("super_bodies,theta", [(0, 0.5), (512, 0.5), (512, 0.3)])
def test_exact_redo_pass_gives_the_same_forces(super_bodies, theta):
    """The exact traversal's second pass: buckets the main pass gives up on (as
    it does when their stacks would outgrow the shared region; forced here on
    every third bucket slot after its first round) are walked again with a
    larger region and get bit-identical forces and the same interaction
    count; the marks are cleared afterwards."""
    from cnb import _lib
    from cnb.core.engine import SimulationEngine
    from cnb.core.state import SimulationState
    from cnb.utils import config as cfgmod
    from cnb.utils.cosmology import zeldovich_arrays
    cfg = cfgmod.make(N_GRID=32, SOFTENING=0.5 / 32, THETA=theta, N_STEPS=100, A_START=0.02,
                      A_END=0.22, KEY_MODE="morton63", FORCE_MODE="grouped", BODIES_PER_LANE=2,
                      BLOCK_WARPS=2, SUPER_BODIES=super_bodies)
    pos, vel = zeldovich_arrays(32, 4)
    st = SimulationState(32 ** 3, pos, vel)
    eng = SimulationEngine(cfg, st, camera=False)
    eng.forces_only()
    eng.check()
    out = []
    for every in (0, 3, 1, 0):
        _lib.call("cnb_exact_test_spill", every)
        try:
            eng.stats.zero_()
            st.force.fill_(float("nan"))
            eng.compute_forces()
            eng.check()
        finally:
            _lib.call("cnb_exact_test_spill", 0)
        tm = eng.tree_manager
        nb = int(tm.workspace[0].item())
        marks = tm.workspace[4:4 + 4 * nb].view(-1, 4)[:, 3]
        assert int(marks.abs().sum().item()) == 0      # every mark cleared by the second pass
        out.append((st.force.cpu().numpy().copy(), int(eng.stats[0].item())))
    f0, c0 = out[0]
    assert np.isfinite(f0).all()
    for f, c in out[1:]:
        np.testing.assert_array_equal(f.view(np.uint32), f0.view(np.uint32))
        assert c == c0
