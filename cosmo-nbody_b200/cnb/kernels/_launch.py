"""Numba-style launch objects: `kernel[grid, block](*args)` or
`kernel[grid, block, stream](*args)`.

The reference launches its kernels with Numba's subscript syntax
(e.g. src/core/state.py:28, src/core/engine.py:95).  These objects accept
the same syntax; the launch shape is validated and recorded (it decides
how many threads exist, which some kernels use as their work count), and
the library chooses its own shape.  The stream is the one given in the
subscript (an int handle, or an object with `.cuda_stream` / `.handle`),
else torch's current stream.
"""
from __future__ import annotations

import functools

from .._arrays import current_stream_ptr


def _dim(x):
    if isinstance(x, int):
        return x
    if isinstance(x, tuple) and x:
        n = 1
        for v in x:
            n *= int(v)
        return n
    raise TypeError(f"invalid launch dimension {x!r}")


def _stream_ptr(s):
    if s is None or s == 0:
        return current_stream_ptr()
    if isinstance(s, int):
        return s
    for attr in ("cuda_stream", "handle", "ptr"):
        v = getattr(s, attr, None)
        if v is not None:
            return int(v.value if hasattr(v, "value") else v)
    raise TypeError(f"unsupported stream object {type(s).__name__}")


class Launch:
    __slots__ = ("grid", "block", "stream", "threads")

    def __init__(self, grid, block, stream):
        self.grid = _dim(grid)
        self.block = _dim(block)
        if self.grid < 0 or self.block <= 0 or self.block > 1024:
            raise ValueError(f"invalid launch configuration [{grid}, {block}]")
        self.threads = self.grid * self.block
        self.stream = _stream_ptr(stream)


class Kernel:
    """A reference-compatible kernel object backed by a libcnb entry point."""

    def __init__(self, name, impl, doc=None):
        self.__name__ = name
        self._impl = impl
        self.__doc__ = doc or impl.__doc__

    def __getitem__(self, cfg):
        if not isinstance(cfg, tuple) or len(cfg) not in (2, 3, 4):
            raise TypeError("launch as kernel[grid, block] or kernel[grid, block, stream]")
        launch = Launch(cfg[0], cfg[1], cfg[2] if len(cfg) > 2 else None)
        return functools.partial(self._impl, launch)

    def __call__(self, *args, **kwargs):
        raise TypeError(f"{self.__name__} is a kernel: launch it as {self.__name__}[grid, block](...)")

    def __repr__(self):
        return f"<cnb kernel {self.__name__}>"
