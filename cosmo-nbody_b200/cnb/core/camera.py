"""Density-splat camera (src/core/camera.py of the reference), on libcnb.

`Camera(n_steps, resolution, config)` and `capture(step, px_d, py_d, pz_d)`
as in the reference (camera.py:10-48): clear the grid, build the orbiting
MVP, splat, colourise.  The grid is [H, W] with W = config.RES_W or
`resolution`, H = config.RES_H or `resolution`; the projection's aspect is
W / H (the reference's square grid gives 1.0).  Frames stay on the device;
the reference's host video buffer, PNG and ffmpeg output
(camera.py:50-70) are not part of this package.
"""
from __future__ import annotations

import torch

from .. import _lib
from ..utils.visualizer import get_mvp_matrix


class Camera:
    def __init__(self, n_steps, resolution, config, device=None):
        self.config = config
        self.n = n_steps
        self.width = int(getattr(config, "RES_W", None) or resolution)
        self.height = int(getattr(config, "RES_H", None) or resolution)
        dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.device = dev
        self.grid_d = torch.zeros((self.height, self.width), dtype=torch.float32, device=dev)
        self.box_center = (config.BOX_SIZE / 2, config.BOX_SIZE / 2, config.BOX_SIZE / 2)
        self.mvp_d = torch.zeros((4, 4), dtype=torch.float32, device=dev)
        # pinned staging for the per-step MVP upload: a copy from pageable memory
        # would stall the host until the stream drains
        self._mvp_pin = [torch.empty((4, 4), dtype=torch.float32).pin_memory() for _ in range(4)]
        self._mvp_ev = [torch.cuda.Event() for _ in range(4)]
        self._mvp_i = 0

    def splat(self, step, px_d, py_d, pz_d):
        """camera.py:40-44: clear, MVP, render_density.  Returns the grid."""
        self.grid_d.zero_()
        mvp = get_mvp_matrix(step, self.box_center, self.config.BOX_SIZE, self.config,
                             aspect=self.width / self.height)
        i = self._mvp_i
        self._mvp_i = (i + 1) % len(self._mvp_pin)
        self._mvp_ev[i].synchronize()          # the upload that last used this buffer has run
        self._mvp_pin[i].copy_(torch.from_numpy(mvp))
        self.mvp_d.copy_(self._mvp_pin[i], non_blocking=True)
        self._mvp_ev[i].record()
        st = int(torch.cuda.current_stream(self.device).cuda_stream)
        _lib.call("cnb_render_density", px_d.data_ptr(), py_d.data_ptr(), pz_d.data_ptr(),
                  self.grid_d.data_ptr(), self.mvp_d.data_ptr(), px_d.shape[0], self.width,
                  self.height, st)
        return self.grid_d

    def mvp_host(self, step):
        """The orbiting camera's MVP for `step` as a pinned host tensor."""
        mvp = get_mvp_matrix(step, self.box_center, self.config.BOX_SIZE, self.config,
                             aspect=self.width / self.height)
        return torch.from_numpy(mvp).pin_memory()

    def splat_device(self, mvp_d, px_d, py_d, pz_d):
        """Clear and splat with an MVP already on the device (no host work, so
        it can be captured in a CUDA graph)."""
        self.grid_d.zero_()
        st = int(torch.cuda.current_stream(self.device).cuda_stream)
        _lib.call("cnb_render_density", px_d.data_ptr(), py_d.data_ptr(), pz_d.data_ptr(),
                  self.grid_d.data_ptr(), mvp_d.data_ptr(), px_d.shape[0], self.width,
                  self.height, st)
        return self.grid_d

    def colorize(self, out_u8=None, out=None):
        """visualizer.py:115-171 on the current grid in two fused kernels;
        returns the float32 [H, W, 3] frame (written to `out` when given, else
        to the camera's own buffer) and fills `out_u8`, uint8 [H, W, 3], with
        the engine.py:139 packing when given."""
        if not hasattr(self, "frame_d"):
            self.frame_d = torch.empty((self.height, self.width, 3), dtype=torch.float32, device=self.device)
            self._cmax = torch.zeros(1, dtype=torch.int32, device=self.device)
        frame = self.frame_d if out is None else out
        st = int(torch.cuda.current_stream(self.device).cuda_stream)
        _lib.call("cnb_colorize", self.grid_d.data_ptr(), self.width, self.height,
                  frame.data_ptr(), out_u8.data_ptr() if out_u8 is not None else None,
                  self._cmax.data_ptr(), st)
        return frame

    def capture(self, step, px_d, py_d, pz_d):
        """camera.py:29-48: splat and colourise; returns the [H, W, 3] frame."""
        self.splat(step, px_d, py_d, pz_d)
        return self.colorize()
