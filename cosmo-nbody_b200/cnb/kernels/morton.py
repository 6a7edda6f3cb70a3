"""Morton keys (src/kernels/morton.py of the reference), on libcnb.

`compute_codes` reproduces the reference's keys bit for bit (its masks keep
the low 10 bits of each 21-bit coordinate, a 30-bit key); `compute_codes_63`
is the full 21-bit interleave (63-bit key) the reference's docstrings
describe, with coordinates clamped to [0, 2^21 - 1].
"""
import numpy as np

from .. import _lib
from .._arrays import dptr, shape_of
from ._launch import Kernel


def _codes_impl(key_mode, launch, pos_x, pos_y, pos_z, codes, indices, n_bodies):
    n = int(n_bodies)
    if n < 0:
        raise ValueError("n_bodies must be >= 0")
    n_arr = shape_of(pos_x)[0]
    n = min(n, n_arr, launch.threads)
    _lib.call("cnb_compute_codes",
              dptr(pos_x, np.float32, (n_arr,), "pos_x"), dptr(pos_y, np.float32, (n_arr,), "pos_y"),
              dptr(pos_z, np.float32, (n_arr,), "pos_z"), dptr(codes, np.uint64, (-1,), "codes"),
              dptr(indices, np.uint32, (-1,), "indices", allow_none=True), n, key_mode,
              launch.stream)


def _compat(launch, pos_x, pos_y, pos_z, codes, indices, n_bodies):
    """morton.py:65-90 compute_codes(pos_x, pos_y, pos_z, codes, indices, n_bodies)."""
    _codes_impl(_lib.KEY_COMPAT30, launch, pos_x, pos_y, pos_z, codes, indices, n_bodies)


def _m63(launch, pos_x, pos_y, pos_z, codes, indices, n_bodies):
    """compute_codes with the full 63-bit key."""
    _codes_impl(_lib.KEY_MORTON63, launch, pos_x, pos_y, pos_z, codes, indices, n_bodies)


compute_codes = Kernel("compute_codes", _compat)
compute_codes_63 = Kernel("compute_codes_63", _m63)

KEY_BITS = {"compat30": 30, "morton63": 63}
KEY_MODES = {"compat30": _lib.KEY_COMPAT30, "morton63": _lib.KEY_MORTON63}
