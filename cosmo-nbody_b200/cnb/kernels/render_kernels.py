"""Density splat (src/kernels/render_kernels.py of the reference), on libcnb.

`render_density(pos_x, pos_y, pos_z, grid, mvp, res)` as in the reference;
a grid of shape [H, W] with W != H is also accepted (the screen mapping then
uses W for x and H for y; the reference's square grid is W = H = res).
"""
import numpy as np

from .. import _lib
from .._arrays import dptr, shape_of
from ._launch import Kernel


def _render(launch, pos_x, pos_y, pos_z, grid, mvp, res):
    """render_kernels.py:12-47 render_density(pos_x, pos_y, pos_z, grid, mvp, res)."""
    n = shape_of(pos_x)[0]
    if launch.threads < n:
        raise ValueError(f"render_density: launch of {launch.threads} threads does not cover {n} bodies")
    h, w = shape_of(grid)
    if h == w and int(res) != w:
        raise ValueError("res must equal the grid size")
    _lib.call("cnb_render_density", dptr(pos_x, np.float32, (n,), "pos_x"),
              dptr(pos_y, np.float32, (n,), "pos_y"), dptr(pos_z, np.float32, (n,), "pos_z"),
              dptr(grid, np.float32, (h, w), "grid"), dptr(mvp, np.float32, (4, 4), "mvp"), n, w, h,
              launch.stream)


render_density = Kernel("render_density", _render)
