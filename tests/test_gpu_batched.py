"""Many boxes in one tree and one persistent launch: every box must get the
forces it would get alone, box subtrees and buckets must not mix boxes, and
a captured CUDA graph must reproduce eager steps bit for bit."""
import numpy as np
import pytest

from oracle import oracle as orc

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


BOXES = [dict(n_grid=8, seed=11, a_start=0.03, theta=0.4),
         dict(n_grid=12, seed=12, a_start=0.05, theta=0.6),
         dict(n_grid=16, seed=13, a_start=0.02, theta=0.5),
         dict(n_grid=10, seed=14, a_start=0.08, theta=0.7)]


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def test_box_roots_and_buckets_respect_boxes():
    from cnb.core.batched import BatchedBoxes
    bb = BatchedBoxes(BOXES)
    bb.sort_and_build()
    roots = host(bb.box_roots)
    ranges = host(bb.ranges)
    n = bb.n
    for b in range(len(BOXES)):
        r = roots[b]
        lo, hi = (r, r) if r < n else tuple(ranges[r - n])
        assert (lo, hi + 1) == (bb.offsets[b], bb.offsets[b + 1])
    bk = host(bb.buckets())
    box_of = np.searchsorted(bb.offsets, bk[:, 0], side="right") - 1
    end_box = np.searchsorted(bb.offsets, bk[:, 0] + bk[:, 1] - 1, side="right") - 1
    np.testing.assert_array_equal(box_of, end_box)
    assert bk[:, 1].sum() == n


def test_batched_theta_zero_is_per_box_direct_sum():
    from cnb import _lib
    from cnb.core.batched import BatchedBoxes
    boxes = [dict(b, theta=1e-6) for b in BOXES]
    bb = BatchedBoxes(boxes)
    bb.sort_and_build()
    bb.compute_forces()
    bb.check()
    f = host(bb.force)
    for b in range(len(boxes)):
        sl = bb.box_slice(b)
        pos = [host(p[sl]) for p in bb.pos]
        mass = host(bb.mass[sl])
        t = np.arange(0, pos[0].size, 5)
        want = orc.direct_sum(*pos, mass, t, 1.0, 0.5 / boxes[b]["n_grid"])
        got = f[sl][t].astype(np.float64)
        e = np.linalg.norm(got - want, axis=1) / np.linalg.norm(want, axis=1)
        assert np.median(e) < 1e-4 and e.max() < 5e-3, (b, np.median(e), e.max())


def test_batched_matches_single_box_runs():
    from cnb.core.batched import BatchedBoxes
    from cnb.core.engine import SimulationEngine
    from cnb.core.state import SimulationState
    from cnb.utils import config as cfgmod
    bb = BatchedBoxes(BOXES, mac="periodic")
    bb.sort_and_build()
    bb.compute_forces()
    f = host(bb.force)
    for b, d in enumerate(BOXES):
        sl = bb.box_slice(b)
        pos = [host(p[sl]) for p in bb.pos]
        vel = [host(v[sl]) for v in bb.vel]
        n = pos[0].size
        cfg = cfgmod.make(N_GRID=d["n_grid"], SOFTENING=0.5 / d["n_grid"], THETA=d["theta"],
                          KEY_MODE="morton63", FORCE_MODE="grouped", MAC="periodic")
        st = SimulationState(n, pos, vel)
        eng = SimulationEngine(cfg, st, camera=False)
        eng.forces_only()
        # the single-box run re-sorts with 63-bit keys: compare body by body
        order = np.lexsort((pos[2], pos[1], pos[0]))
        sp = [host(p) for p in st.pos]
        order2 = np.lexsort((sp[2], sp[1], sp[0]))
        single = host(st.force)[order2]
        batched = f[sl][order]
        scale = np.abs(single).max()
        assert np.median(np.abs(single - batched).max(axis=1)) <= 1e-5 * scale


def test_integrate_boxes_matches_oracle():
    from cnb.core.batched import BatchedBoxes
    bb = BatchedBoxes(BOXES)
    bb.sort_and_build()
    rng = np.random.default_rng(0)
    F = torch.from_numpy((rng.standard_normal((bb.n, 3)) * 3).astype(np.float32)).cuda()
    bb.force.copy_(F)
    before = [host(p) for p in bb.pos + bb.vel]
    a0 = host(bb.a).copy()
    bb.integrate()
    after = [host(p) for p in bb.pos + bb.vel]
    for b in range(len(BOXES)):
        sl = bb.box_slice(b)
        a = a0[b]
        H = orc.hubble(a)
        dt = 0.002 / (a * H) * 0.8
        want = orc.integrate(*(x[sl] for x in before), host(F)[sl], a, H, dt)
        for got, w in zip(after, want):
            np.testing.assert_array_equal(got[sl], w)
    np.testing.assert_allclose(host(bb.a), a0 + 0.002, rtol=0, atol=1e-15)


def test_graph_replay_equals_eager_steps():
    from cnb.core.batched import BatchedBoxes
    eager = BatchedBoxes(BOXES)
    graphed = BatchedBoxes(BOXES)
    graphed.capture(warmup=1)        # 1 eager warm-up step, captured graph = 2 steps
    eager.step()
    for _ in range(2):
        graphed.replay()
        eager.step()
        eager.step()
    torch.cuda.synchronize()
    for a, b in zip(eager.pos + eager.vel, graphed.pos + graphed.vel):
        np.testing.assert_array_equal(host(a), host(b))
    np.testing.assert_array_equal(host(eager.a), host(graphed.a))
    eager.check()
    graphed.check()
