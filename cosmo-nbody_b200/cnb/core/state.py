"""Particle state (src/core/state.py of the reference), on libcnb.

`SimulationState(n_bodies, pos_init, vel_init)` keeps the reference's
attributes: `pos` and `vel` (3-tuples of float32 device arrays, SoA), `force`
[N,3], `mass` (1/N), `codes` (uint64), `indices` (uint32).  Inputs may be
torch tensors, numpy arrays or any CUDA array; float64 inputs (the
reference's main.py passes float64 CuPy arrays) are converted to float32
once, here.

`sort_buffer_by_morton(config)` computes the keys (config.KEY_MODE,
"compat30" by default = the reference's keys), sorts (key, index) pairs with
libcnb's stable radix sort and gathers positions, velocities and masses.
config.SORT_MODE picks the sort: "full" (the radix sort every step),
"adaptive" (the near-sorted path first: keys that were sorted one step
earlier mostly keep their order; the result is the same argsort) or "auto"
(adaptive for "morton63" keys, full for "compat30" keys, whose low 10 bits
per axis reorder at every step).
Like the reference it rebinds `pos`, `vel`, `mass` and `codes` to the sorted
arrays; the arrays alternate between two preallocated sets, so no memory is
allocated per step.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from .. import _lib
from .._arrays import status_buffer
from ..kernels.morton import KEY_BITS, KEY_MODES


SORT_MODES = {"full": _lib.SORT_FULL, "adaptive": _lib.SORT_ADAPTIVE}


def sort_mode_for(config, key_mode):
    """The SORT_MODES name config.SORT_MODE selects for keys of key_mode."""
    mode = getattr(config, "SORT_MODE", "auto")
    if mode == "auto":
        return "adaptive" if key_mode == "morton63" else "full"
    if mode not in SORT_MODES:
        raise ValueError(f"SORT_MODE must be 'auto', 'full' or 'adaptive', got {mode!r}")
    return mode


def _to_device_f32(a, device):
    if isinstance(a, torch.Tensor):
        return a.to(device=device, dtype=torch.float32).contiguous()
    if hasattr(a, "__cuda_array_interface__"):
        return torch.as_tensor(a, device=device).to(torch.float32).contiguous()
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to(device)


class SortContext:
    """Owns the libcnb scratch for sorting up to n_max keys."""

    def __init__(self, n_max):
        self.ptr = C.c_void_p()
        _lib.call("cnb_ctx_create", int(n_max), C.byref(self.ptr))
        self.n_max = int(n_max)

    def sort_pairs(self, keys_in, keys_out, idx_in, perm_out, n, key_bits, stream, status=None):
        """Stable (key, index) sort; the sort's device flags are ORed into
        `status` (the shared device status word when None)."""
        _lib.call("cnb_sort_pairs", self.ptr, keys_in, keys_out, idx_in, perm_out, int(n),
                  int(key_bits), stream)
        if status is None:
            status = status_buffer().data_ptr()
        _lib.call("cnb_ctx_take_flags", self.ptr, status, stream)

    def set_mode(self, mode):
        """SORT_MODES name: "full" radix sort every call, or "adaptive"
        (near-sorted path first, full sort only when it does not apply)."""
        _lib.call("cnb_ctx_set_sort_mode", self.ptr, SORT_MODES[mode])

    def stats(self):
        """(sorts that took the near-sorted path, full radix sorts run);
        synchronises the device."""
        out = (C.c_int64 * 2)()
        _lib.call("cnb_ctx_sort_stats", self.ptr, out)
        return int(out[0]), int(out[1])

    def close(self):
        if self.ptr:
            _lib.load().cnb_ctx_destroy(self.ptr)
            self.ptr = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class SimulationState:
    """state.py:5-18 SimulationState(n_bodies, pos_init, vel_init)."""

    def __init__(self, n_bodies, pos_init, vel_init, device=None):
        self.n = int(n_bodies)
        dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.device = dev
        self.pos = tuple(_to_device_f32(p, dev) for p in pos_init)
        self.vel = tuple(_to_device_f32(v, dev) for v in vel_init)
        for a in self.pos + self.vel:
            if a.shape != (self.n,):
                raise ValueError(f"state arrays must have shape ({self.n},), got {tuple(a.shape)}")
        self.force = torch.zeros((self.n, 3), dtype=torch.float32, device=dev)
        self.mass = torch.full((self.n,), 1.0 / self.n if self.n else 0.0, dtype=torch.float32, device=dev)
        self.codes = torch.zeros(self.n, dtype=torch.uint64, device=dev)
        # morton.py:90 writes indices[i] = i; the reference never reads them back
        self.indices = torch.arange(self.n, dtype=torch.int64, device=dev).to(torch.uint32)
        # second buffer set for the permutation gathers
        self._alt = [torch.empty(self.n, dtype=torch.float32, device=dev) for _ in range(7)]
        self._codes_alt = torch.empty(self.n, dtype=torch.uint64, device=dev)
        self.perm = torch.empty(self.n, dtype=torch.uint32, device=dev)
        self._ctx = None

    def _stream(self):
        return int(torch.cuda.current_stream(self.device).cuda_stream)

    def compute_codes(self, key_mode="compat30"):
        """morton.py:65-90 over the current state (writes self.codes, self.indices)."""
        p = self.pos
        _lib.call("cnb_compute_codes", p[0].data_ptr(), p[1].data_ptr(), p[2].data_ptr(),
                  self.codes.data_ptr(), self.indices.data_ptr(), self.n, KEY_MODES[key_mode],
                  self._stream())

    def sort_buffer_by_morton(self, config):
        """state.py:20-40: keys, stable argsort, gathers of pos/vel/mass/codes."""
        key_mode = getattr(config, "KEY_MODE", "compat30")
        if self.n == 0:
            return
        if self._ctx is None:
            self._ctx = SortContext(self.n)
        self._ctx.set_mode(sort_mode_for(config, key_mode))
        st = self._stream()
        p = self.pos
        _lib.call("cnb_compute_codes", p[0].data_ptr(), p[1].data_ptr(), p[2].data_ptr(),
                  self.codes.data_ptr(), None, self.n, KEY_MODES[key_mode], st)
        self._ctx.sort_pairs(self.codes.data_ptr(), self._codes_alt.data_ptr(), None,
                             self.perm.data_ptr(), self.n, KEY_BITS[key_mode], st)
        src = list(self.pos) + list(self.vel) + [self.mass]
        dst = self._alt
        src_arr = (C.c_void_p * 7)(*[t.data_ptr() for t in src])
        dst_arr = (C.c_void_p * 7)(*[t.data_ptr() for t in dst])
        _lib.call("cnb_gather_f32", self.perm.data_ptr(), 7, src_arr, dst_arr, self.n, st)
        self.pos = tuple(dst[0:3])
        self.vel = tuple(dst[3:6])
        self.mass = dst[6]
        self._alt = src
        self.codes, self._codes_alt = self._codes_alt, self.codes
