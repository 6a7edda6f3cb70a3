"""Float64 Ewald sums for the periodic force law (test infrastructure only).

No reference counterpart: the reference applies the minimum-image force
(physics_kernels.py:118-141).  This is the periodic law the library's
"ewald" opening test approximates, written from the standard Ewald
decomposition of a periodic lattice of point masses with a uniform
neutralising background (unit box, G = 1, unit source mass):

  f_per(d) = sum_n  d_n / r_n^3 * [erfc(a r_n) + (2 a r_n / sqrt(pi)) exp(-a^2 r_n^2)]
           + 4 pi sum_{k != 0} k / k^2 * exp(-k^2 / (4 a^2)) * sin(k . d)

with d = source - target, d_n = d - n over lattice vectors n, k = 2 pi m.
It is the acceleration of the target towards the source and all its images.
Near d = 0 it behaves as d / |d|^3 - (4 pi / 3) d; the rest,

  g(d) = f_per(d) - d / |d|^3 + (4 pi / 3) d,

is smooth, odd and of order |d|^3.
"""
from __future__ import annotations

import math

import numpy as np

ALPHA = 2.0
N_REAL = 3      # real-space images with |n_i| <= N_REAL
N_RECIP = 4     # reciprocal vectors with |m_i| <= N_RECIP
LINEAR = 4.0 * math.pi / 3.0


def _lattice(k):
    r = np.arange(-k, k + 1, dtype=np.float64)
    g = np.stack(np.meshgrid(r, r, r, indexing="ij"), -1).reshape(-1, 3)
    return g


_REAL = _lattice(N_REAL)
_RECIP = _lattice(N_RECIP)
_RECIP = _RECIP[np.any(_RECIP != 0, axis=1)] * (2.0 * math.pi)
_RECIP_W = 4.0 * math.pi * np.exp(-np.sum(_RECIP ** 2, 1) / (4 * ALPHA ** 2)) / np.sum(_RECIP ** 2, 1)


def _erfc(x):
    from scipy.special import erfc
    return erfc(x)


def f_per(d, alpha=ALPHA):
    """Periodic acceleration towards a unit mass at displacement d (float64 [..., 3])."""
    d = np.asarray(d, dtype=np.float64)
    shape = d.shape
    d = d.reshape(-1, 3)
    out = np.zeros_like(d)
    for n in _REAL:
        dn = d - n
        r = np.sqrt(np.sum(dn * dn, 1))
        with np.errstate(divide="ignore", invalid="ignore"):
            w = (_erfc(alpha * r) + 2 * alpha * r / math.sqrt(math.pi) * np.exp(-(alpha * r) ** 2)) / r ** 3
        w[r == 0] = 0.0
        out += dn * w[:, None]
    w_k = 4.0 * math.pi * np.exp(-np.sum(_RECIP ** 2, 1) / (4 * alpha ** 2)) / np.sum(_RECIP ** 2, 1)
    out += np.sin(d @ _RECIP.T) @ (_RECIP * w_k[:, None])
    return out.reshape(shape)


def g_corr(d, alpha=ALPHA):
    """g(d) = f_per(d) - d/|d|^3 + (4 pi/3) d (smooth; 0 at d = 0)."""
    d = np.asarray(d, dtype=np.float64)
    r = np.sqrt(np.sum(d * d, -1, keepdims=True))
    with np.errstate(divide="ignore", invalid="ignore"):
        mono = np.where(r > 0, d / r ** 3, 0.0)
    return f_per(d, alpha) - mono + LINEAR * d


def min_image(d):
    return d - np.round(d)


def direct_sum_ewald(px, py, pz, mass, targets, G, soft):
    """Float64 periodic direct sum for the targets: per pair the softened
    monopole at the minimum image (with the reference's d^2 > 1e-7 cut) plus
    the periodic correction f_per(d) - d/|d|^3 of that image."""
    p = np.stack([np.asarray(a, np.float64) for a in (px, py, pz)], 1)
    m = np.asarray(mass, np.float64)
    out = np.zeros((len(targets), 3))
    for t, i in enumerate(targets):
        d = min_image(p - p[i])
        d2 = np.sum(d * d, 1)
        keep = d2 > 1e-7
        dk = d[keep]
        mono = dk / (d2[keep] + soft * soft)[:, None] ** 1.5
        corr = g_corr(dk) - LINEAR * dk
        out[t] = G * np.sum(m[keep][:, None] * (mono + corr), 0)
    return out
