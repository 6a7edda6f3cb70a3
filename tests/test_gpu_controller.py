"""Learned opening-angle controller: GPU gradients against the CPU oracle,
the fused bfloat16 inference against the oracle network, training, labels
from the batched boxes, and the gain over plain fixed theta."""
import numpy as np
import pytest

from oracle import mlp

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def st():
    return int(torch.cuda.current_stream().cuda_stream)


def test_gpu_gradient_matches_oracle():
    from cnb import _lib
    rng = np.random.default_rng(0)
    p = (rng.standard_normal(mlp.N_PARAMS) * 0.3).astype(np.float32)
    n = 1000
    X = rng.standard_normal((n, mlp.N_IN)).astype(np.float32)
    y = rng.uniform(0.2, 1.0, n).astype(np.float32)
    P, Xd, yd = (torch.from_numpy(a).cuda() for a in (p, X, y))
    scratch = torch.empty(4 * 64 * n + n, device="cuda")
    g = torch.empty(mlp.N_PARAMS, device="cuda")
    loss = torch.zeros(1, device="cuda")
    _lib.call("cnb_mlp_grad", Xd.data_ptr(), yd.data_ptr(), n, P.data_ptr(), 3.0, scratch.data_ptr(),
              g.data_ptr(), loss.data_ptr(), st())
    wl, wg = mlp.loss_and_grad(p.astype(np.float64), X, y, over_weight=3.0)
    gg = g.cpu().numpy()
    assert abs(loss.item() - wl) <= 1e-5 * max(1.0, wl)
    np.testing.assert_allclose(gg, wg, rtol=0, atol=2e-4 * np.abs(wg).max())
    # per block of parameters, the relative error is small too
    for lo, hi in ((mlp.OFF_W1, mlp.OFF_B1), (mlp.OFF_W2, mlp.OFF_B2), (mlp.OFF_W3, mlp.OFF_B3)):
        rel = np.linalg.norm(gg[lo:hi] - wg[lo:hi]) / np.linalg.norm(wg[lo:hi])
        assert rel < 1e-4, (lo, rel)


@pytest.mark.parametrize("n", [1000, 1003, 70000])
def test_tensor_core_gradient_matches_oracle(n):
    """cnb_mlp_grad_mma (bf16 tensor-core contractions, float32 accumulation)
    against the float64 oracle with the same operands rounded to bf16, and
    against the exact float64 gradient; n not a multiple of 32 pads with
    samples of zero gradient."""
    from cnb import _lib
    rng = np.random.default_rng(7)
    p = (rng.standard_normal(mlp.N_PARAMS) * 0.3).astype(np.float32)
    X = rng.standard_normal((n, mlp.N_IN)).astype(np.float32)
    y = rng.uniform(0.2, 1.0, n).astype(np.float32)
    P, Xd, yd = (torch.from_numpy(a).cuda() for a in (p, X, y))
    nbytes = int(_lib.load().cnb_mlp_grad_mma_scratch_bytes(n))
    assert nbytes >= 208 * 2 * n
    scratch = torch.empty(nbytes // 4 + 4, device="cuda")
    g = torch.full((mlp.N_PARAMS,), 7.0, device="cuda")   # overwritten, not accumulated into
    loss = torch.full((1,), 7.0, device="cuda")
    _lib.call("cnb_mlp_grad_mma", Xd.data_ptr(), yd.data_ptr(), n, P.data_ptr(), 3.0,
              scratch.data_ptr(), nbytes, g.data_ptr(), loss.data_ptr(), st())
    gg = g.cpu().numpy().astype(np.float64)
    tl, tg = mlp.loss_and_grad_tc(p.astype(np.float64), X, y, over_weight=3.0)
    el, eg = mlp.loss_and_grad(p.astype(np.float64), X, y, over_weight=3.0)
    assert abs(loss.item() - tl) <= 1e-5 * max(1.0, tl)
    for lo, hi in ((mlp.OFF_W1, mlp.OFF_B1), (mlp.OFF_B1, mlp.OFF_W2), (mlp.OFF_W2, mlp.OFF_B2),
                   (mlp.OFF_B2, mlp.OFF_W3), (mlp.OFF_W3, mlp.OFF_B3), (mlp.OFF_B3, mlp.N_PARAMS)):
        rel_tc = np.linalg.norm(gg[lo:hi] - tg[lo:hi]) / np.linalg.norm(tg[lo:hi])
        rel_ex = np.linalg.norm(gg[lo:hi] - eg[lo:hi]) / np.linalg.norm(eg[lo:hi])
        assert rel_tc < 2e-3, (lo, rel_tc)      # the same bf16 operands: float32 sums only
        assert rel_ex < 3e-2, (lo, rel_ex)      # bf16 operands against exact float64
    with pytest.raises(_lib.CnbError):
        _lib.call("cnb_mlp_grad_mma", Xd.data_ptr(), yd.data_ptr(), n, P.data_ptr(), 3.0,
                  scratch.data_ptr(), nbytes - 16, g.data_ptr(), loss.data_ptr(), st())


def test_predict_matches_oracle_forward():
    from cnb import _lib
    rng = np.random.default_rng(1)
    p = (rng.standard_normal(mlp.N_PARAMS) * 0.3).astype(np.float32)
    X = rng.standard_normal((513, mlp.N_IN)).astype(np.float32)
    out = torch.empty(513, device="cuda")
    P, Xd = torch.from_numpy(p).cuda(), torch.from_numpy(X).cuda()
    _lib.call("cnb_mlp_predict", Xd.data_ptr(), 513, P.data_ptr(), out.data_ptr(), st())
    want, _ = mlp.forward(p, X)
    np.testing.assert_allclose(out.cpu().numpy(), want, rtol=0, atol=1e-5)


def _built_engine(n_grid=16, seed=2):
    from cnb.core.engine import SimulationEngine
    from cnb.core.state import SimulationState
    from cnb.utils import config as cfgmod
    from cnb.utils.cosmology import zeldovich_arrays
    cfg = cfgmod.make(N_GRID=n_grid, SOFTENING=0.5 / n_grid, THETA=0.5, KEY_MODE="morton63",
                      FORCE_MODE="grouped", MAC="periodic")
    pos, vel = zeldovich_arrays(n_grid, seed)
    eng = SimulationEngine(cfg, SimulationState(n_grid ** 3, pos, vel), camera=False)
    eng.forces_only()
    return eng


def test_features_and_fused_inference_match_oracle():
    from cnb.controller import ThetaController, bucket_features
    eng = _built_engine()
    tm = eng.tree_manager
    n = eng.state.n
    # accelerations of a step with a permutation as the previous-step input
    acc = eng.state.force.clone()
    perm = torch.from_numpy(np.random.default_rng(9).permutation(n).astype(np.uint32)).cuda()
    feats = bucket_features(tm.node_table, tm.parent, tm.workspace, n, acc, perm).cpu().numpy()
    flat = tm.node_table.cpu().numpy().reshape(-1, 4)   # 2M records then 2M boxes
    m = flat.shape[0] // 4
    rec = flat[:2 * m].reshape(m, 2, 4)
    aabb = flat[2 * m:].reshape(m, 2, 4)
    parents = tm.parent.cpu().numpy()
    bk = tm.workspace[4:4 + 4 * feats.shape[0]].view(-1, 4).cpu().numpy()
    acc_h, perm_h = acc.cpu().numpy(), perm.cpu().numpy()
    want = np.stack([mlp.bucket_features(rec, aabb, parents, b, acc_h, perm_h) for b in bk])
    np.testing.assert_allclose(feats, want, rtol=1e-4, atol=1e-4)
    ctl = ThetaController(seed=3)
    ctl.mean = torch.from_numpy(want.mean(0).astype(np.float32)).cuda()
    ctl.std = torch.from_numpy(want.std(0).astype(np.float32) + 1e-3).cuda()
    th = ctl.theta_for_buckets(tm.node_table, tm.parent, tm.workspace, n, acc,
                               perm)[:feats.shape[0]].cpu().numpy()
    folded = mlp.bf16_round(ctl.folded_params().cpu().numpy())
    wth, _ = mlp.forward(folded, feats, hidden_bf16=True)
    np.testing.assert_allclose(th, wth, rtol=0, atol=2e-4)
    # the float32-hidden network differs only by that rounding
    wth32, _ = mlp.forward(folded, feats)
    assert np.abs(th - wth32).max() < 5e-3


def test_training_fits_a_smooth_target():
    from cnb.controller import ThetaController
    rng = np.random.default_rng(4)
    X = rng.standard_normal((4000, 12)).astype(np.float32)
    y = (0.6 + 0.3 * np.tanh(X[:, 0] - 0.5 * X[:, 3])).astype(np.float32)
    ctl = ThetaController(seed=5)
    curve = ctl.train(torch.from_numpy(X), torch.from_numpy(y), steps=600, lr=3e-3, over_weight=1.0)
    assert curve[-1] < 0.1 * curve[0]
    pred = ctl.predict(torch.from_numpy(X)).cpu().numpy()
    assert np.sqrt(np.mean((pred - y) ** 2)) < 0.05


def test_labels_and_learned_theta_gain():
    """Train on labels from a batch of small boxes, then compare with plain
    theta = 0.5 on a held-out box at matched 99th-percentile error
    (RMS-normalised, float64 direct sum).  Under the exact minimum-image
    opening test most of the work (sources near the planes antipodal to a
    bucket) does not depend on theta; the comparison is on the part that does
    (interactions not needing the per-pair image, stats[0] - stats[2])."""
    from cnb.controller import ThetaController, make_labels, direct_sum
    from cnb.core.batched import BatchedBoxes, draw_boxes
    train = BatchedBoxes(draw_boxes(16, seed=3, grids=(16, 24, 32)), mac="periodic")
    X, y, info = make_labels(train, per_box=96, error="rms")
    assert info["n_samples"] > 500 and 0 < info["budget"] < 1
    ctl = ThetaController(seed=0)
    ctl.train(X, y, steps=1500, lr=3e-3, over_weight=4.0)
    eng = _built_engine(n_grid=32, seed=77)          # held-out box
    s = eng.state
    eng.controller_accel = s.force.clone()           # the features' acceleration input, fixed
    t = torch.from_numpy(np.sort(np.random.default_rng(0).choice(s.n, 4096, replace=False))).cuda()
    ref = direct_sum(s.pos, s.mass, t, 1.0, eng.config.SOFTENING)
    rms = ref.norm(dim=1).pow(2).mean().sqrt()

    def run(scale=None):
        eng.controller = ctl if scale is not None else None
        eng.controller_scale = scale or 1.0
        if scale is None:
            eng.theta_per_group = None
        eng.stats.zero_()
        eng.compute_forces()
        e = ((s.force[t].double() - ref).norm(dim=1) / rms).cpu().numpy()
        st_ = eng.stats.cpu().numpy()
        return float(np.percentile(e, 99)), float(st_[0] - st_[2]) / s.n

    p99_plain, cost_plain = run(None)
    lo, hi = 0.3, 3.0        # global scale of the learned angles matched to the plain error
    for _ in range(14):
        mid = 0.5 * (lo + hi)
        p99, _ = run(mid)
        lo, hi = (mid, hi) if p99 <= p99_plain else (lo, mid)
    p99_l, cost_l = run(lo)
    eng.controller = None
    eng.check()
    gain = cost_plain / cost_l
    print(f"plain: p99 {p99_plain:.4g} theta-dependent work {cost_plain:.0f}/body; "
          f"learned: p99 {p99_l:.4g} work {cost_l:.0f}/body (scale {lo:.3f}); "
          f"gain {gain:.3f}x; labels {info}")
    # the calibrated controller meets the plain method's error ...
    assert p99_l <= p99_plain * 1.001
    # ... and its work is reported as the gain.  On these near-uniform states
    # the labels are close to uniform and the measured gain is about 0.9x
    # (no gain); the bound only guards against a broken controller.
    assert gain > 0.7, (cost_l, cost_plain, p99_l, p99_plain)


def test_lagrangian_labels_and_gain_under_the_periodic_law():
    """Under the periodic (Ewald) law, where theta sets the cost: labels from
    the Lagrangian allocation of a batch of small boxes (least interactions
    at plain theta = 0.5's p99), the network trained on them, and on a
    held-out 48^3 box the learned angles -- scaled to plain's p99 relative
    error against the float64 Ewald direct sum -- need fewer interactions
    than plain theta = 0.5.  The allocation's own gain on the training
    buckets is the bound of any per-bucket policy there."""
    from cnb.controller import ThetaController, make_labels, direct_sum
    from cnb.core.batched import BatchedBoxes, draw_boxes
    from cnb.core.engine import SimulationEngine
    from cnb.core.state import SimulationState
    from cnb.utils import config as cfgmod
    from cnb.utils.cosmology import zeldovich_arrays
    train = BatchedBoxes(draw_boxes(16, seed=3, grids=(16, 24, 32)), mac="ewald", bodies_per_lane=2)
    X, y, info = make_labels(train, per_box=512)
    assert info["objective"] == "lagrangian"
    assert info["violations"] <= info["allowed_violations"]
    assert info["bound"] > 1.2
    ctl = ThetaController(seed=0)
    ctl.train(X, y, steps=1500, lr=3e-3, over_weight=2.0)
    n_grid = 48
    cfg = cfgmod.make(N_GRID=n_grid, SOFTENING=0.5 / n_grid, THETA=0.5, KEY_MODE="morton63",
                      FORCE_MODE="grouped", MAC="ewald", BODIES_PER_LANE=2, BLOCK_WARPS=4)
    pos, vel = zeldovich_arrays(n_grid, 77)
    eng = SimulationEngine(cfg, SimulationState(n_grid ** 3, pos, vel), camera=False)
    eng.forces_only()
    acc = eng.state.force.clone()
    s = eng.state
    t = torch.from_numpy(np.sort(np.random.default_rng(0).choice(s.n, 1024, replace=False))).cuda()
    ref = direct_sum(s.pos, s.mass, t, 1.0, cfg.SOFTENING, periodic=True)

    def run(scale=None):
        eng.controller = ctl if scale is not None else None
        eng.controller_scale = scale or 1.0
        eng.controller_accel = acc
        if scale is None:
            eng.theta_per_group = None
        eng.stats.zero_()
        eng.compute_forces()
        e = ((s.force[t].double() - ref).norm(dim=1) / ref.norm(dim=1)).cpu().numpy()
        return float(np.percentile(e, 99)), float(eng.stats[0].item()) / s.n

    p99_plain, cost_plain = run(None)
    lo, hi = 0.2, 3.0
    for _ in range(14):
        mid = 0.5 * (lo + hi)
        p99, _ = run(mid)
        lo, hi = (mid, hi) if p99 <= p99_plain else (lo, mid)
    p99_l, cost_l = run(lo)
    eng.controller = None
    eng.check()
    gain = cost_plain / cost_l
    print(f"periodic law: plain p99 {p99_plain:.4g} {cost_plain:.0f}/body; learned p99 {p99_l:.4g} "
          f"{cost_l:.0f}/body (scale {lo:.3f}); gain {gain:.3f}x; label bound {info['bound']:.3f}x")
    assert p99_l <= p99_plain
    assert gain > 1.15, (gain, info)
