"""HostStepper: host-fed steps with the copies on their own streams give the
same results as copy-in, step, copy-out one after another, for every
submission of a stream of them (positions and velocities bit for bit; the
density grid to float32 atomic order)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _engine(n_grid, seed):
    from cnb.core.engine import SimulationEngine
    from cnb.core.state import SimulationState
    from cnb.utils import config as cfgmod
    from cnb.utils.cosmology import zeldovich_arrays
    cfg = cfgmod.make(N_GRID=n_grid, SOFTENING=0.5 / n_grid, THETA=0.5, N_STEPS=10, A_START=0.02,
                      A_END=0.04, KEY_MODE="morton63", FORCE_MODE="grouped", BODIES_PER_LANE=2,
                      BLOCK_WARPS=4, RES=256, RES_W=320, RES_H=200)
    pos, vel = zeldovich_arrays(n_grid, seed)
    return SimulationEngine(cfg, SimulationState(n_grid ** 3, pos, vel)), pos, vel


def test_pipelined_submissions_match_serial_steps():
    from cnb.core.hoststep import HostStepper
    n_grid, steps = 32, 5
    n = n_grid ** 3
    eng_a, pos, vel = _engine(n_grid, 3)
    eng_b, _, _ = _engine(n_grid, 3)
    rng = np.random.default_rng(0)
    # a different host state per submission: the ICs with small seeded shifts
    inputs = []
    for k in range(steps):
        arrs = [np.mod(np.asarray(a) + rng.normal(0, 1e-4, n), 1.0).astype(np.float32) for a in pos]
        arrs += [np.asarray(v, np.float32) * (1 + 0.1 * k) for v in vel]
        inputs.append([torch.from_numpy(a).pin_memory() for a in arrs])
    outs = [[torch.empty(n, dtype=torch.float32).pin_memory() for _ in range(6)] for _ in range(steps)]
    shape = tuple(eng_a.camera.grid_d.shape)
    grids = [torch.empty(shape, dtype=torch.float32).pin_memory() for _ in range(steps)]
    hs = HostStepper(eng_a)
    for k in range(steps):
        hs.submit(inputs[k], outs[k], grids[k])
    hs.synchronize()
    eng_a.check()
    s = eng_b.state
    for k in range(steps):
        for d, h in zip(s.pos + s.vel, inputs[k]):
            d.copy_(h.cuda())
        eng_b.step()
        g = eng_b.camera.splat(k, *s.pos)
        torch.cuda.synchronize()
        for d, h in zip(s.pos + s.vel, outs[k]):
            np.testing.assert_array_equal(h.numpy(), d.cpu().numpy())
        np.testing.assert_allclose(grids[k].numpy(), g.cpu().numpy(), rtol=1e-5, atol=1e-6)
    eng_b.check()


def test_rejects_pageable_or_misshapen_host_arrays():
    from cnb.core.hoststep import HostStepper
    eng, _, _ = _engine(8, 1)
    hs = HostStepper(eng)
    n = eng.state.n
    good = [torch.empty(n, dtype=torch.float32).pin_memory() for _ in range(6)]
    with pytest.raises(ValueError):
        hs.submit([torch.empty(n, dtype=torch.float32) for _ in range(6)], good)
    with pytest.raises(ValueError):
        hs.submit(good[:5], good)
    with pytest.raises(ValueError):
        hs.submit(good, [torch.empty(n + 1, dtype=torch.float32).pin_memory() for _ in range(6)])
