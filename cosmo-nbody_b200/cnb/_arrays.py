"""Device-array plumbing for the drop-in kernels.

Accepts anything exposing ``__cuda_array_interface__`` (torch CUDA tensors,
CuPy arrays, Numba device arrays).  Host arrays are rejected: the reference's
kernels only ever receive device arrays.
"""
from __future__ import annotations

import numpy as np
import torch

from ._lib import CnbError, FLAG_BAD_TOPOLOGY, FLAG_LIST_OVERFLOW, FLAG_NONFINITE, \
    FLAG_SORT_CHECK, FLAG_STACK_OVERFLOW, FLAG_WAIT_LIMIT

_TYPESTR = {
    np.dtype(np.float32): "<f4",
    np.dtype(np.float64): "<f8",
    np.dtype(np.int32): "<i4",
    np.dtype(np.int64): "<i8",
    np.dtype(np.uint32): "<u4",
    np.dtype(np.uint64): "<u8",
}


def cai(arr):
    """Return the __cuda_array_interface__ dict of `arr` or raise TypeError."""
    iface = getattr(arr, "__cuda_array_interface__", None)
    if iface is None:
        raise TypeError(f"expected a CUDA device array, got {type(arr).__name__}")
    return iface


def dptr(arr, dtype, shape=None, name="array", allow_none=False):
    """Device pointer of a C-contiguous array with the given dtype (and
    shape, where a dimension of -1 matches anything)."""
    if arr is None:
        if allow_none:
            return None
        raise TypeError(f"{name}: expected a device array, got None")
    iface = cai(arr)
    want = np.dtype(dtype)
    got = np.dtype(iface["typestr"])
    if got != want:
        raise TypeError(f"{name}: dtype {got} where {want} is required")
    shp = tuple(iface["shape"])
    if shape is not None:
        if len(shp) != len(shape) or any(s != -1 and s != g for s, g in zip(shape, shp)):
            raise ValueError(f"{name}: shape {shp} where {tuple(shape)} is required")
    strides = iface.get("strides")
    if strides is not None:
        expect = []
        acc = got.itemsize
        for d in reversed(shp):
            expect.append(acc)
            acc *= d
        expect = tuple(reversed(expect))
        if any(d > 1 and s != e for d, s, e in zip(shp, strides, expect)):
            raise ValueError(f"{name}: must be C-contiguous")
    return int(iface["data"][0])


def shape_of(arr):
    return tuple(cai(arr)["shape"])


def device_of(arr):
    """CUDA device index of `arr`."""
    if isinstance(arr, torch.Tensor):
        return arr.device.index if arr.device.index is not None else torch.cuda.current_device()
    return torch.cuda.current_device()


def current_stream_ptr(device=None):
    return int(torch.cuda.current_stream(device).cuda_stream)


_status = {}


def status_buffer(device=None):
    """One int32 status word per device, shared by the drop-in kernels."""
    dev = torch.cuda.current_device() if device is None else device
    buf = _status.get(dev)
    if buf is None:
        buf = torch.zeros(1, dtype=torch.int32, device=f"cuda:{dev}")
        _status[dev] = buf
    return buf


FLAG_NAMES = {
    FLAG_STACK_OVERFLOW: "traversal stack overflow (children dropped)",
    FLAG_BAD_TOPOLOGY: "invalid tree topology",
    FLAG_NONFINITE: "non-finite acceleration",
    FLAG_LIST_OVERFLOW: "grouped traversal work queue exhausted",
    FLAG_WAIT_LIMIT: "a bounded wait between blocks gave up (sort result invalid)",
    FLAG_SORT_CHECK: "a destination check of the near-sorted sort failed (sort result invalid)",
}


def describe_flags(flags):
    return ", ".join(v for k, v in FLAG_NAMES.items() if flags & k) or "none"


def read_status(device=None, clear=True):
    """Synchronise and return (then clear) the device status word."""
    buf = status_buffer(device)
    val = int(buf.item())
    if clear and val:
        buf.zero_()
    return val


def check_status(device=None,
                 fatal=FLAG_BAD_TOPOLOGY | FLAG_NONFINITE | FLAG_LIST_OVERFLOW | FLAG_WAIT_LIMIT |
                       FLAG_SORT_CHECK):
    """Raise CnbError if a fatal flag was raised since the last check."""
    val = read_status(device)
    if val & fatal:
        raise CnbError(f"device status: {describe_flags(val)}", flags=val)
    return val
