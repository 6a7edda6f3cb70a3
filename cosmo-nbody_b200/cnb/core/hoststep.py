"""Host-fed steps with the transfers under the compute (no counterpart in the
reference, whose state lives in device memory for the whole run).

`HostStepper(engine)` steps states that live in pinned host memory:
`submit(host_in, host_out, grid_out=None)` copies the six float32 arrays
(x, y, z, vx, vy, vz) of `host_in` into the engine's state, runs
`engine.step()` (and the density splat of the new positions when `grid_out`
is given), and copies the stepped arrays to `host_out` (and the grid to
`grid_out`).  It returns at once: submissions go through two staging slots,
and the copy-in of submission k + 1 and the copy-out of submission k run on
their own streams while the device computes, so a stream of submissions costs
about max(compute, transfers) per step instead of their sum.  Every
submission still moves all of its bytes across PCIe.  `synchronize()` waits
until every submitted copy-out has landed in host memory; the host arrays of a
submission must not be touched before that.

Per submission: 24 bytes per body in, 24 bytes per body (+ 4 per grid pixel)
out, plus two device-to-device copies between the staging slots and the
engine's state (the state arrays alternate inside the step).
"""
from __future__ import annotations

import torch


class HostStepper:
    def __init__(self, engine):
        self.eng = engine
        st = engine.state
        dev = st.device
        n = st.n
        f32 = dict(dtype=torch.float32, device=dev)
        self.slots_in = [[torch.empty(n, **f32) for _ in range(6)] for _ in range(2)]
        self.slots_out = [[torch.empty(n, **f32) for _ in range(6)] for _ in range(2)]
        cam = engine.camera
        self.grids = [torch.empty(tuple(cam.grid_d.shape), **f32) for _ in range(2)] if cam else None
        self.h2d = torch.cuda.Stream(dev)
        self.d2h = torch.cuda.Stream(dev)
        ev = lambda: [torch.cuda.Event() for _ in range(2)]  # noqa: E731
        self.in_ready, self.in_free, self.out_ready, self.out_free = ev(), ev(), ev(), ev()
        self.k = 0

    @staticmethod
    def _check(host, n, what):
        if len(host) != 6:
            raise ValueError(f"{what}: six arrays (x, y, z, vx, vy, vz)")
        for h in host:
            if h.dtype != torch.float32 or h.device.type != "cpu" or h.shape != (n,):
                raise ValueError(f"{what}: float32 host tensors of shape ({n},)")
            if not h.is_pinned():
                raise ValueError(f"{what}: host tensors must be pinned (copies are asynchronous)")

    def submit(self, host_in, host_out, grid_out=None):
        eng, st = self.eng, self.eng.state
        self._check(host_in, st.n, "host_in")
        self._check(host_out, st.n, "host_out")
        if grid_out is not None:
            if self.grids is None:
                raise ValueError("grid_out needs an engine with a camera")
            if grid_out.shape != self.grids[0].shape or not grid_out.is_pinned():
                raise ValueError(f"grid_out: pinned float32 host tensor of shape "
                                 f"{tuple(self.grids[0].shape)}")
        s = self.k % 2
        main = torch.cuda.current_stream(st.device)
        # copy in (waits until the step that last used this slot has read it)
        with torch.cuda.stream(self.h2d):
            if self.k >= 2:
                self.h2d.wait_event(self.in_free[s])
            for d, h in zip(self.slots_in[s], host_in):
                d.copy_(h, non_blocking=True)
            self.in_ready[s].record(self.h2d)
        main.wait_event(self.in_ready[s])
        for d, src in zip(st.pos + st.vel, self.slots_in[s]):
            d.copy_(src)
        self.in_free[s].record(main)
        eng.step()
        grid = eng.camera.splat(self.k, *st.pos) if grid_out is not None else None
        # copy out (waits until the copy-out that last used this slot is done)
        if self.k >= 2:
            main.wait_event(self.out_free[s])
        for d, src in zip(self.slots_out[s], st.pos + st.vel):
            d.copy_(src)
        if grid is not None:
            self.grids[s].copy_(grid)
        self.out_ready[s].record(main)
        with torch.cuda.stream(self.d2h):
            self.d2h.wait_event(self.out_ready[s])
            for h, d in zip(host_out, self.slots_out[s]):
                h.copy_(d, non_blocking=True)
            if grid is not None:
                grid_out.copy_(self.grids[s], non_blocking=True)
            self.out_free[s].record(self.d2h)
        self.k += 1

    def synchronize(self):
        """Waits for every submitted copy-out (and everything before it)."""
        self.d2h.synchronize()
        torch.cuda.current_stream(self.eng.state.device).synchronize()
