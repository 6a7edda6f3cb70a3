"""Zel'dovich initial conditions and the Hubble rate
(src/utils/cosmology.py of the reference).

The recipe is the reference's (cosmology.py:27-71): P(k) ~ k^-2.5 with the DC
term removed, uniform random phases, displacement = Re ifftn(i k / k^2
delta_k) rescaled to a standard deviation of 0.3 / n_grid, positions
(grid + d) mod 1, velocities d * H(a0) * Omega_m(a0)^0.55 * a0 / 20.  The
phases come from numpy's PCG64 generator seeded with `seed` (the reference
seeds CuPy's generator with 42, a stream numpy cannot reproduce), so every
path -- GPU, CPU baseline, tests -- is fed the same arrays.  Output is
float32 (the reference keeps float64; the B200 step stores float32).
"""
from __future__ import annotations

import numpy as np


def get_hubble_param(a, config):
    """cosmology.py:76-84: H0 sqrt(Omega_m a^-3 + Omega_L)."""
    return config.H0 * np.sqrt(config.OMEGA_M * a ** -3 + config.OMEGA_L)


def zeldovich_arrays(n_grid, seed, a_start=0.02, H0=67.8, omega_m=1.0, omega_l=0.692):
    """(pos [3][N] float32, vel [3][N] float32) on an n_grid^3 lattice, N = n_grid^3."""
    n = int(n_grid)
    rng = np.random.default_rng(seed)
    k = np.fft.fftfreq(n) * n
    kx = k[:, None, None]
    ky = k[None, :, None]
    kz = k[None, None, :]
    k2 = kx * kx + ky * ky + kz * kz
    k_mag = np.sqrt(k2)
    k_mag[0, 0, 0] = 1e-10
    P = k_mag ** -2.5
    P[0, 0, 0] = 0.0
    phase = rng.uniform(0.0, 2.0 * np.pi, (n, n, n))
    delta_k = np.sqrt(P) * (np.cos(phase) + 1j * np.sin(phase))
    del phase, P
    denom = k_mag ** 2 + 1e-10

    def disp(kc):
        term = 1j * np.broadcast_to(kc, (n, n, n)) / denom
        term[0, 0, 0] = 0.0
        return np.fft.ifftn(term * delta_k).real.ravel()

    d = [disp(kx), disp(ky), disp(kz)]
    scale = (1.0 / n) * 0.3 / np.std(d[0])
    d = [di * scale for di in d]
    lin = np.linspace(0.0, 1.0, n, endpoint=False)
    g = np.meshgrid(lin, lin, lin, indexing="ij")
    pos = []
    for gi, di in zip(g, d):
        p = ((gi.ravel() + di) % 1.0).astype(np.float32)
        p[p >= np.float32(1.0)] = np.float32(0.0)  # float32 rounding of values just below 1
        pos.append(p)
    H_start = H0 * np.sqrt(omega_m * a_start ** -3 + omega_l)
    om_a = omega_m * a_start ** -3 / (omega_m * a_start ** -3 + omega_l)
    coupling = H_start * om_a ** 0.55 * a_start / 20.0
    vel = [(di * coupling).astype(np.float32) for di in d]
    return pos, vel


def zeldovich_tensors(n_grid, seed, device, a_start=0.02, H0=67.8, omega_m=1.0, omega_l=0.692):
    """zeldovich_arrays with the field work on `device` (torch; cuFFT on a
    GPU): the same seeded phases (numpy PCG64, drawn on the host), then the
    spectrum, the three inverse FFTs, the normalisation and the lattice sum
    in float64 on the device.  Returns float32 tensors ([pos x, y, z],
    [vel x, y, z]) equal to zeldovich_arrays' to float32 rounding (the FFTs
    differ in the last float64 bits)."""
    import torch
    n = int(n_grid)
    dev = torch.device(device)
    f64 = torch.float64
    rng = np.random.default_rng(seed)
    phase = torch.from_numpy(rng.uniform(0.0, 2.0 * np.pi, (n, n, n))).to(dev)
    k = torch.fft.fftfreq(n, device=dev, dtype=f64) * n
    kx, ky, kz = k.view(n, 1, 1), k.view(1, n, 1), k.view(1, 1, n)
    k_mag = torch.sqrt(kx * kx + ky * ky + kz * kz)
    k_mag[0, 0, 0] = 1e-10
    P = k_mag ** -2.5
    P[0, 0, 0] = 0.0
    delta_k = torch.sqrt(P) * torch.complex(torch.cos(phase), torch.sin(phase))
    del phase, P
    denom = k_mag ** 2 + 1e-10
    d = []
    for kc in (kx, ky, kz):
        term = torch.complex(torch.zeros((), dtype=f64, device=dev), kc.expand(n, n, n) / denom)
        term[0, 0, 0] = 0.0
        d.append(torch.fft.ifftn(term * delta_k).real.reshape(-1))
        del term
    del delta_k
    scale = (1.0 / n) * 0.3 / torch.std(d[0], correction=0)
    d = [di * scale for di in d]
    lin = torch.arange(n, device=dev, dtype=f64) * (1.0 / n)
    g = torch.meshgrid(lin, lin, lin, indexing="ij")
    pos = []
    for gi, di in zip(g, d):
        p = torch.remainder(gi.reshape(-1) + di, 1.0).to(torch.float32)
        p[p >= 1.0] = 0.0  # float32 rounding of values just below 1
        pos.append(p)
    H_start = H0 * np.sqrt(omega_m * a_start ** -3 + omega_l)
    om_a = omega_m * a_start ** -3 / (omega_m * a_start ** -3 + omega_l)
    coupling = H_start * om_a ** 0.55 * a_start / 20.0
    vel = [(di * coupling).to(torch.float32) for di in d]
    return pos, vel


def generate_zeldovich_ics(config, seed=None, device=None):
    """cosmology.py:12-73 generate_zeldovich_ics(config).  Returns
    ([pos_x, pos_y, pos_z], [vel_x, vel_y, vel_z]) as float32 numpy arrays, or
    float32 torch tensors on `device` when given (the field is then built on
    that device, zeldovich_tensors)."""
    seed = getattr(config, "SEED", 0) if seed is None else seed
    if device is not None:
        return zeldovich_tensors(config.N_GRID, seed, device, config.A_START, config.H0,
                                 config.OMEGA_M, config.OMEGA_L)
    return zeldovich_arrays(config.N_GRID, seed, config.A_START, config.H0, config.OMEGA_M,
                            config.OMEGA_L)


def density_contrast_sigma(px, py, pz, grid=64):
    """Standard deviation of the density contrast on a grid^3 count mesh (a
    clustering diagnostic for evolved states)."""
    ix = np.minimum((np.asarray(px) * grid).astype(np.int64), grid - 1)
    iy = np.minimum((np.asarray(py) * grid).astype(np.int64), grid - 1)
    iz = np.minimum((np.asarray(pz) * grid).astype(np.int64), grid - 1)
    counts = np.bincount((ix * grid + iy) * grid + iz, minlength=grid ** 3).astype(np.float64)
    mean = counts.mean()
    return float(np.std(counts / mean - 1.0)) if mean > 0 else 0.0
