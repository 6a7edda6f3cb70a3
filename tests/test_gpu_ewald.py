"""Periodic (Ewald) force law: the float64 table of g and its Jacobian, the
float64 Ewald direct-sum oracle, and the grouped traversal's "ewald" test
against that oracle.  The correction of every accepted node is taken to
first order about the bucket centre, so its error grows with the square of
the bucket size relative to the box: the accuracy tests use 32^3 bodies."""
import math

import numpy as np
import pytest

from oracle import ewald as E
from oracle import oracle as orc

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _stream():
    return int(torch.cuda.current_stream().cuda_stream)


def _table(nt):
    from cnb import _lib
    t = torch.empty(((nt + 1) ** 3, 24), dtype=torch.float32, device="cuda")
    _lib.call("cnb_ewald_table", t.data_ptr(), nt, _stream())
    torch.cuda.synchronize()
    return t


def _jac(d, h=1e-4):
    out = np.zeros(d.shape + (3,))
    for j in range(3):
        e = np.zeros(3)
        e[j] = h
        out[..., :, j] = (E.g_corr(d + e) - E.g_corr(d - e)) / (2 * h)
    return out


def test_table_matches_float64_restatement():
    nt = 8
    t = _table(nt).cpu().numpy().astype(np.float64)
    h = 0.5 / nt
    ijk = np.stack(np.meshgrid(*(np.arange(nt + 1),) * 3, indexing="ij"), -1).reshape(-1, 3)
    d = ijk * h
    g = E.g_corr(d)
    np.testing.assert_allclose(t[:, 0:3], g, rtol=1e-5, atol=1e-6)
    assert np.abs(t[:, 3]).max() == 0.0
    # the Jacobian (xx, xy, xz, yy, yz, zz); g is O(|d|^3), so it vanishes at 0
    J = np.zeros((len(d), 3, 3))
    nz = np.any(ijk > 0, 1)
    J[nz] = _jac(d[nz])
    want = np.stack([J[:, 0, 0], J[:, 0, 1], J[:, 0, 2], J[:, 1, 1], J[:, 1, 2], J[:, 2, 2]], 1)
    got = np.concatenate([t[:, 4:8], t[:, 8:10]], 1)
    np.testing.assert_allclose(got, want, rtol=1e-5, atol=2e-5)
    # second derivatives H_ijk = d J_ij / d d_k (xxx, xxy, xxz, xyy, xyz, xzz, yyy, yyz, yzz, zzz)
    sel = np.nonzero(nz)[0][::7]
    H = np.zeros((len(sel), 3, 3, 3))
    hstep = 1e-3
    for k in range(3):
        e = np.zeros(3)
        e[k] = hstep
        H[:, :, :, k] = (_jac(d[sel] + e) - _jac(d[sel] - e)) / (2 * hstep)
    idx = [(0, 0, 0), (0, 0, 1), (0, 0, 2), (0, 1, 1), (0, 1, 2), (0, 2, 2), (1, 1, 1), (1, 1, 2),
           (1, 2, 2), (2, 2, 2)]
    want_h = np.stack([H[:, i, j, k] for i, j, k in idx], 1)
    got_h = np.concatenate([t[sel, 12:16], t[sel, 16:20], t[sel, 20:22]], 1)
    np.testing.assert_allclose(got_h, want_h, rtol=1e-3, atol=2e-3)
    assert np.abs(t[:, 22:24]).max() == 0.0


def test_direct_sum_kernel_matches_restatement():
    from cnb import _lib
    rng = np.random.default_rng(4)
    n = 300
    p = rng.random((n, 3)).astype(np.float32)
    m = np.full(n, 1.0 / n, np.float32)
    targets = np.array([0, 7, 111, 299], np.int64)
    P = [torch.from_numpy(np.ascontiguousarray(p[:, i])).cuda() for i in range(3)]
    M = torch.from_numpy(m).cuda()
    T = torch.from_numpy(targets).cuda()
    out = torch.empty((len(targets), 3), dtype=torch.float64, device="cuda")
    _lib.call("cnb_direct_sum_ewald_f64", *(q.data_ptr() for q in P), M.data_ptr(), n, T.data_ptr(),
              len(targets), 1.0, 0.02, out.data_ptr(), _stream())
    want = E.direct_sum_ewald(p[:, 0], p[:, 1], p[:, 2], m, targets, 1.0, 0.02)
    np.testing.assert_allclose(out.cpu().numpy(), want, rtol=1e-9, atol=1e-12)


def _sorted_bodies(n_grid, seed):
    from cnb.utils.cosmology import zeldovich_arrays
    (x, y, z), _ = zeldovich_arrays(n_grid, seed)
    codes, _ = orc.compute_codes(x, y, z, 1)
    perm = orc.argsort_stable(codes)
    return [a[perm] for a in (x, y, z)], codes[perm]


class Tree:
    def __init__(self, pos, codes, bpl=2, quad=False):
        from cnb.core.octree import OctreeManager
        self.n = n = codes.size
        self.P = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in pos]
        self.M = torch.full((n,), 1.0 / n, device="cuda")
        self.bpl = bpl
        self.tm = OctreeManager(n, node_table=True, bucket=32 * bpl, quad=quad)
        self.tm.build(self.P, self.M, torch.from_numpy(codes).cuda())
        self.table = _table(64)

    def forces(self, theta, soft):
        from cnb import _lib
        f = torch.empty((self.n, 3), device="cuda")
        stats = torch.zeros(4, dtype=torch.int64, device="cuda")
        status = torch.zeros(1, dtype=torch.int32, device="cuda")
        _lib.call("cnb_forces_grouped_ewald", *(p.data_ptr() for p in self.P),
                  self.tm.node_table.data_ptr(), self.tm.workspace.data_ptr(), f.data_ptr(), self.n,
                  theta, None, self.bpl, 4, 1.0, soft, self.table.data_ptr(), 64,
                  self.tm.quad.data_ptr() if self.tm.quad is not None else None, None, None, stats.data_ptr(),
                  status.data_ptr(), _stream())
        torch.cuda.synchronize()
        assert int(status.item()) == 0
        return f.cpu().numpy().astype(np.float64), stats.cpu().numpy()

    def oracle(self, targets, soft):
        from cnb import _lib
        T = torch.from_numpy(np.asarray(targets, np.int64)).cuda()
        out = torch.empty((len(targets), 3), dtype=torch.float64, device="cuda")
        _lib.call("cnb_direct_sum_ewald_f64", *(p.data_ptr() for p in self.P), self.M.data_ptr(), self.n,
                  T.data_ptr(), len(targets), 1.0, soft, out.data_ptr(), _stream())
        return out.cpu().numpy()


def _errors(f, ref):
    rms = np.sqrt(np.mean(np.sum(ref ** 2, 1)))
    e = np.linalg.norm(f - ref, axis=1)
    return np.median(e / np.linalg.norm(ref, axis=1)), np.percentile(e / rms, 99)


def test_theta_zero_equals_periodic_direct_sum():
    pos, codes = _sorted_bodies(32, 5)
    tr = Tree(pos, codes)
    soft = 0.5 / 32
    f, stats = tr.forces(0.0, soft)
    assert int(stats[0]) == tr.n * tr.n
    t = np.random.default_rng(0).choice(tr.n, 256, replace=False)
    med, p99 = _errors(f[t], tr.oracle(t, soft))
    # only the first-order correction about the bucket centre is approximate
    # (measured at this size: median 4.2e-3, p99 1.7e-2; it falls as the
    # square of the bucket size)
    assert med < 8e-3 and p99 < 3e-2, (med, p99)


def test_theta_half_accuracy_and_cost():
    pos, codes = _sorted_bodies(32, 6)
    tr = Tree(pos, codes)
    soft = 0.5 / 32
    f, stats = tr.forces(0.5, soft)
    t = np.random.default_rng(1).choice(tr.n, 256, replace=False)
    med, p99 = _errors(f[t], tr.oracle(t, soft))
    per_body = stats[0] / tr.n
    print(f"ewald theta=0.5: median rel {med:.2e}, p99 rms {p99:.2e}, {per_body:.0f} interactions/body")
    assert med < 4e-2 and p99 < 8e-2, (med, p99)   # measured: 2.1e-2, 4.4e-2
    assert per_body < 0.3 * tr.n        # far from the direct sum
    # a smaller theta is more accurate
    f2, _ = tr.forces(0.3, soft)
    med2, _ = _errors(f2[t], tr.oracle(t, soft))
    assert med2 < med


def test_theta_zero_matches_restated_bucket_algorithm():
    """At theta = 0 every leaf is accepted, so the kernel's result can be
    restated exactly on the CPU from its bucket table: per bucket the centre
    of the bodies' box, per source the image nearest that centre, per pair
    the softened monopole of that image, per body -(4 pi/3) m (c - x) and
    the table's g and Jacobian at the nearest grid point, to first order."""
    pos, codes = _sorted_bodies(8, 9)
    tr = Tree(pos, codes, bpl=1)
    soft = 0.5 / 8
    f, _ = tr.forces(0.0, soft)
    want = _restated_theta_zero(tr, pos, soft)
    scale = np.sqrt(np.mean(np.sum(want ** 2, 1)))
    assert np.abs(f - want).max() < 2e-4 * scale, np.abs(f - want).max() / scale


def _close_pair_bodies(n_grid, seed):
    """Zel'dovich bodies with companions planted next to 40 of them at
    distances on both sides of the reference's cut d^2 > 1e-7 (one coincident)."""
    from cnb.utils.cosmology import zeldovich_arrays
    (x, y, z), _ = zeldovich_arrays(n_grid, seed)
    p = np.stack([x, y, z], 1).astype(np.float64)
    rng = np.random.default_rng(seed + 11)
    idx = rng.choice(np.arange(0, p.shape[0] - 1, 2), 40, replace=False)
    dist = np.array([0.0, 1e-4, 2.5e-4, 3.0e-4, 3.4e-4, 4e-4, 1e-3])
    for k, i in enumerate(idx):
        u = rng.normal(size=3)
        p[i + 1] = p[i] + dist[k % dist.size] * u / np.linalg.norm(u)
    x, y, z = (np.mod(p[:, k], 1.0).astype(np.float32) for k in range(3))
    codes, _ = orc.compute_codes(x, y, z, 1)
    perm = orc.argsort_stable(codes)
    return [a[perm] for a in (x, y, z)], codes[perm]


@pytest.mark.parametrize("bpl,quad", [(1, False), (2, False), (2, True)])
def test_theta_zero_close_pairs_honour_the_cut(bpl, quad):
    """Without quadrupoles the cut is tested only on entries near each
    bucket's box (the second list); with them, on the first list as a whole.
    With softening 1e-4 a pair inside the cut would dominate the force
    of its bodies if it were applied; the kernel must match the restatement,
    which applies the cut to every pair."""
    pos, codes = _close_pair_bodies(8, 3)
    tr = Tree(pos, codes, bpl=bpl, quad=quad)
    soft = 1e-4
    f, _ = tr.forces(0.0, soft)
    want = _restated_theta_zero(tr, pos, soft)
    scale = np.sqrt(np.mean(np.sum(want ** 2, 1)))
    assert np.abs(f - want).max() < 2e-4 * scale, np.abs(f - want).max() / scale


def _restated_theta_zero(tr, pos, soft):
    T = tr.table.cpu().numpy().astype(np.float64)
    nt = 64
    p = np.stack(pos, 1).astype(np.float64)
    m = 1.0 / tr.n
    ws = tr.tm.workspace.cpu().numpy()
    want = np.zeros((tr.n, 3))
    for b in range(int(ws[0])):
        lo, cnt = ws[4 + 4 * b], ws[5 + 4 * b]
        body = p[lo:lo + cnt].astype(np.float32)
        centre = (0.5 * (body.min(0) + body.max(0))).astype(np.float64)
        dc = p - centre
        dc -= np.where(dc > 0.5, 1.0, np.where(dc < -0.5, -1.0, 0.0))
        a = np.abs(dc)
        ijk = np.minimum(np.rint(a * 2 * nt).astype(np.int64), nt)
        t = (ijk[:, 0] * (nt + 1) + ijk[:, 1]) * (nt + 1) + ijk[:, 2]
        e = a - ijk / (2 * nt)
        g0, j0 = T[t, 0:3], T[t, 4:10]
        Jo = np.stack([np.stack([j0[:, 0], j0[:, 1], j0[:, 2]], 1),
                       np.stack([j0[:, 1], j0[:, 3], j0[:, 4]], 1),
                       np.stack([j0[:, 2], j0[:, 4], j0[:, 5]], 1)], 1)
        sgn = np.where(dc < 0, -1.0, 1.0)
        g = sgn * (g0 + np.einsum("nij,nj->ni", Jo, e))
        J = Jo * sgn[:, :, None] * sgn[:, None, :]
        for i in range(lo, lo + cnt):
            d = centre + dc - p[i]
            d2 = np.sum(d * d, 1)
            keep = d2 > 1e-7
            mono = d[keep] / (d2[keep] + soft * soft)[:, None] ** 1.5
            corr = -4 * math.pi / 3 * d + g + np.einsum("nij,j->ni", J, centre - p[i])
            want[i] = m * (mono.sum(0) + corr.sum(0))
    return want


def test_correction_error_falls_with_bucket_size():
    """At theta = 0 the only approximation is the correction taken to first
    order about each bucket centre: 32-body buckets beat 64-body ones."""
    pos, codes = _sorted_bodies(32, 5)
    soft = 0.5 / 32
    t = np.random.default_rng(0).choice(32 ** 3, 256, replace=False)
    meds = []
    for bpl in (2, 1):
        tr = Tree(pos, codes, bpl=bpl)
        f, _ = tr.forces(0.0, soft)
        meds.append(_errors(f[t], tr.oracle(t, soft))[0])
    assert meds[1] < 0.85 * meds[0], meds


def test_engine_runs_the_periodic_law():
    from cnb.core.engine import SimulationEngine
    from cnb.core.state import SimulationState
    from cnb.utils import config as cfgmod
    from cnb.utils.cosmology import zeldovich_arrays
    cfg = cfgmod.make(N_GRID=16, SOFTENING=0.5 / 16, THETA=0.5, N_STEPS=10, A_START=0.02, A_END=0.04,
                      KEY_MODE="morton63", FORCE_MODE="grouped", MAC="ewald", BODIES_PER_LANE=2,
                      BLOCK_WARPS=4)
    pos, vel = zeldovich_arrays(16, 2)
    st = SimulationState(16 ** 3, pos, vel)
    eng = SimulationEngine(cfg, st, camera=False)
    for _ in range(3):
        eng.step()
    eng.check()
    p = np.stack([t.cpu().numpy() for t in st.pos])
    assert np.all((p >= 0) & (p <= 1)) and np.isfinite(st.force.cpu().numpy()).all()
    with pytest.raises(ValueError):
        eng.set_super_bodies(512)


def test_batched_boxes_follow_the_periodic_law_per_box():
    """Several boxes in one launch: each box is periodic on its own unit cube
    and its forces match the same box run alone through the engine."""
    from cnb.core.batched import BatchedBoxes
    from cnb.core.engine import SimulationEngine
    from cnb.core.state import SimulationState
    from cnb.utils import config as cfgmod
    from cnb.utils.cosmology import zeldovich_arrays
    boxes = [dict(n_grid=16, seed=1, a_start=0.02, theta=0.5), dict(n_grid=24, seed=2, a_start=0.05, theta=0.6),
             dict(n_grid=16, seed=3, a_start=0.08, theta=0.4)]
    bb = BatchedBoxes(boxes, mac="ewald", bodies_per_lane=1)
    bb.sort_and_build()
    bb.compute_forces()
    bb.check()
    for b, d in enumerate(boxes):
        sl = bb.box_slice(b)
        got = bb.force[sl].cpu().numpy().astype(np.float64)
        pb = np.stack([bb.pos[k][sl].cpu().numpy() for k in range(3)], 1)
        cfg = cfgmod.make(N_GRID=d["n_grid"], SOFTENING=0.5 / d["n_grid"], THETA=d["theta"], N_STEPS=10,
                          A_START=d["a_start"], A_END=d["a_start"] + 0.02, KEY_MODE="morton63",
                          FORCE_MODE="grouped", MAC="ewald", BODIES_PER_LANE=1, BLOCK_WARPS=4)
        pos, vel = zeldovich_arrays(d["n_grid"], d["seed"], d["a_start"])
        st = SimulationState(d["n_grid"] ** 3, pos, vel)
        eng = SimulationEngine(cfg, st, camera=False)
        eng.forces_only()
        eng.check()
        # the engine sorted its own copy: match bodies by position
        pe = np.stack([p.cpu().numpy() for p in st.pos], 1)
        fe = st.force.cpu().numpy().astype(np.float64)
        order_b = np.lexsort(pb.T)
        order_e = np.lexsort(pe.T)
        np.testing.assert_array_equal(pb[order_b], pe[order_e])
        diff = np.linalg.norm(got[order_b] - fe[order_e], axis=1)
        rms = np.sqrt(np.mean(np.sum(fe ** 2, 1)))
        assert np.median(diff) < 1e-3 * rms and np.percentile(diff, 99) < 0.05 * rms, \
            (np.median(diff) / rms, np.percentile(diff, 99) / rms)


def test_upward_second_moments_match_direct_sums():
    """cnb_upward_table_quad: every internal node's second central moment
    equals the one summed directly over its bodies (a node of a Karras tree
    covers a contiguous range of the sorted bodies); the traversal table is
    the one the monopole pass writes."""
    from cnb import _lib
    from cnb.core.octree import OctreeManager
    pos, codes = _sorted_bodies(16, 3)
    n = codes.size
    P = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in pos]
    M = torch.full((n,), 1.0 / n, device="cuda")
    K = torch.from_numpy(codes).cuda()
    tq = OctreeManager(n, node_table=True, quad=True)
    tq.build(P, M, K)
    t0 = OctreeManager(n, node_table=True)
    t0.build(P, M, K)
    torch.cuda.synchronize()
    # the same table, except that internal nodes carry b_max in the 3-D-extent slot
    a_, b_ = tq.node_table.cpu().numpy(), t0.node_table.cpu().numpy()
    rec_q, rec_0 = a_[0:2].reshape(-1, 2, 4), b_[0:2].reshape(-1, 2, 4)
    np.testing.assert_array_equal(a_[2:], b_[2:])
    np.testing.assert_array_equal(rec_q[:, 0], rec_0[:, 0])
    np.testing.assert_array_equal(rec_q[:, 1, [0, 2, 3]], rec_0[:, 1, [0, 2, 3]])
    np.testing.assert_array_equal(rec_q[:n, 1, 1], rec_0[:n, 1, 1])
    q = tq.quad.cpu().numpy().astype(np.float64)
    rg = tq.ranges.cpu().numpy()
    p = np.stack(pos, 1).astype(np.float64)
    rng = np.random.default_rng(0)
    for i in rng.choice(n - 1, 400, replace=False):
        lo, hi = int(rg[i, 0]), int(rg[i, 1])
        b = p[lo:hi + 1]
        m = 1.0 / n
        c = b.mean(0)
        s = b - c
        M2 = m * s.T @ s
        want = np.array([M2[0, 0], M2[0, 1], M2[0, 2], M2[1, 1], M2[1, 2], M2[2, 2]])
        got = np.concatenate([q[n + i, 0:4], q[n + i, 4:6]])
        scale = m * (hi - lo + 1) * np.max(np.sum(s * s, 1))
        np.testing.assert_allclose(got, want, rtol=0, atol=2e-5 * scale + 1e-30)
        # b_max bounds every member's distance from the CoM
        bmax = float(rec_q[n + i, 1, 1])
        assert np.sqrt(np.max(np.sum(s * s, 1))) <= bmax * (1 + 1e-5) + 1e-7


def test_quadrupoles_lower_the_error():
    from cnb.core.octree import OctreeManager
    pos, codes = _sorted_bodies(32, 6)
    soft = 0.5 / 32
    tm = Tree(pos, codes)
    f_mono, s_mono = tm.forces(0.5, soft)
    tq = Tree.__new__(Tree)
    tq.__dict__.update(tm.__dict__)
    tq.tm = OctreeManager(tm.n, node_table=True, bucket=64, quad=True)
    tq.tm.build(tm.P, tm.M, torch.from_numpy(codes).cuda())
    f_quad, s_quad = tq.forces(0.5, soft)
    # quadrupole mode opens on b_max (<= the 3-D extent's diagonal): fewer interactions
    assert int(s_quad[2]) > 0
    t = np.random.default_rng(1).choice(tm.n, 256, replace=False)
    ref = tm.oracle(t, soft)
    mm, pm = _errors(f_mono[t], ref)
    mq, pq = _errors(f_quad[t], ref)
    print(f"theta 0.5 monopole: median {mm:.2e} p99 {pm:.2e} ({s_mono[0] / tm.n:.0f}/body); "
          f"quadrupole: median {mq:.2e} p99 {pq:.2e} ({s_quad[0] / tm.n:.0f}/body)")
    # at the same theta: no worse than monopoles, with far fewer interactions
    assert mq < mm and pq < pm and s_quad[0] < 0.7 * s_mono[0], (mm, mq, pm, pq)
    # theta = 0 accepts leaves only: no quadrupole entries; the monopole mode's
    # second list holds the leaves near each bucket's box (the cut's), which the
    # quadrupole mode applies from its first list; the same forces up to rounding
    f0, s0 = tq.forces(0.0, soft)
    g0, sg = tm.forces(0.0, soft)
    assert int(s0[2]) == 0 and 0 < int(sg[2]) < int(sg[0])
    scale = np.sqrt(np.mean(np.sum(g0 ** 2, 1)))
    # float32 sums of 32 768 terms in two orders
    assert np.abs(f0 - g0).max() < 1e-4 * scale
