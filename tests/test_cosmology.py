"""Initial conditions: the torch form of the Zel'dovich generator (the one a
GPU runs through cuFFT) gives the numpy generator's arrays bit for bit when
run on the CPU (both use pocketfft there)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")


@pytest.mark.parametrize("n,seed", [(8, 0), (16, 3), (32, 1)])
def test_torch_generator_equals_numpy_generator(n, seed):
    from cnb.utils.cosmology import zeldovich_arrays, zeldovich_tensors
    pos, vel = zeldovich_arrays(n, seed)
    pos_t, vel_t = zeldovich_tensors(n, seed, "cpu")
    for a, b in zip(pos + vel, pos_t + vel_t):
        assert b.dtype == torch.float32 and b.shape == (n ** 3,)
        np.testing.assert_array_equal(a, b.numpy())
    p = np.stack([t.numpy() for t in pos_t])
    assert np.all((p >= 0) & (p < 1))


def test_generate_ics_dispatch():
    from cnb.utils import config as cfgmod
    from cnb.utils.cosmology import generate_zeldovich_ics
    cfg = cfgmod.make(N_GRID=8, SEED=2)
    pos, vel = generate_zeldovich_ics(cfg)
    assert isinstance(pos[0], np.ndarray)
    pos_t, vel_t = generate_zeldovich_ics(cfg, device="cpu")
    np.testing.assert_array_equal(pos[1], pos_t[1].numpy())
    np.testing.assert_array_equal(vel[2], vel_t[2].numpy())
