"""Many independent periodic boxes of uneven size stepped as one (no
reference counterpart: the reference simulates a single box).

All boxes' bodies live in one set of arrays, box after box.  Keys carry the
box id in their top bits (cnb_compute_codes_boxes), so one radix sort and one
Karras build give every box its own subtree; the upward pass is the usual
one; the grouped traversal runs every bucket against its own box's subtree
with that box's (theta, softening) in one persistent launch; the integrator
reads each box's (a, H, dt) from device memory.  Because nothing in a step
depends on host values, the whole step can be captured once in a CUDA graph
and replayed (`capture()` / `replay()`).

Within a box the bodies are re-sorted every step, but each box keeps its
range [offset_b, offset_b + n_b) of the arrays, so box ids and masses never
move.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from .. import _lib
from .._arrays import check_status, status_buffer
from ..utils.cosmology import zeldovich_arrays
from .state import SortContext

MACS = {"ref_x": _lib.MAC_REF_X, "ref_x_bucket": _lib.MAC_REF_X_BUCKET,
        "periodic": _lib.MAC_PERIODIC, "ewald": _lib.MAC_EWALD}
EWALD_NT = 64


def draw_boxes(n_boxes=64, seed=3, grids=(16, 24, 32, 48, 64), a_range=(0.02, 0.1),
               theta_range=(0.3, 0.8)):
    """Box descriptors of the uneven-box workload: n_grid drawn uniformly from
    `grids`, a_start from `a_range`, theta from `theta_range` (seeded)."""
    rng = np.random.default_rng(seed)
    out = []
    for b in range(n_boxes):
        out.append(dict(n_grid=int(rng.choice(grids)), seed=int(seed * 1000 + b),
                        a_start=float(rng.uniform(*a_range)),
                        theta=float(rng.uniform(*theta_range))))
    return out


class BatchedBoxes:
    """Independent boxes in one tree.  `boxes` is a list of dicts with keys
    n_grid, seed, a_start, theta (see draw_boxes)."""

    def __init__(self, boxes, mac="periodic", bodies_per_lane=1, block_warps=4, da=0.002, G=1.0,
                 H0=67.8,
                 omega_m=1.0, omega_l=0.692, slab_bodies=0.0, device=None):
        dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.device = dev
        self.boxes = boxes
        self.n_boxes = len(boxes)
        self.box_bits = max(1, math.ceil(math.log2(max(self.n_boxes, 2))))
        if self.box_bits > 30:
            raise ValueError("too many boxes")
        self.mac = MACS[mac]
        self.bpl = int(bodies_per_lane)
        self.block_warps = int(block_warps)
        self.da, self.G = float(da), float(G)
        self.H0, self.omega_m, self.omega_l = H0, omega_m, omega_l
        sizes = [b["n_grid"] ** 3 for b in boxes]
        self.sizes = np.array(sizes, np.int64)
        self.offsets = np.concatenate([[0], np.cumsum(self.sizes)]).astype(np.int64)
        n = int(self.offsets[-1])
        self.n = n
        pos = [np.empty(n, np.float32) for _ in range(3)]
        vel = [np.empty(n, np.float32) for _ in range(3)]
        mass = np.empty(n, np.float32)
        box_id = np.empty(n, np.int32)
        params = np.zeros((self.n_boxes, 4), np.float32)
        for b, d in enumerate(boxes):
            lo, hi = self.offsets[b], self.offsets[b + 1]
            p, v = zeldovich_arrays(d["n_grid"], d["seed"], d["a_start"], H0, omega_m, omega_l)
            for k in range(3):
                pos[k][lo:hi] = p[k]
                vel[k][lo:hi] = v[k]
            mass[lo:hi] = 1.0 / (hi - lo)
            box_id[lo:hi] = b
            params[b] = (d["theta"], 0.5 / d["n_grid"], slab_bodies / (hi - lo), 0.0)
        t = lambda a: torch.from_numpy(a).to(dev)
        self.pos = [t(a) for a in pos]
        self.vel = [t(a) for a in vel]
        self.mass = t(mass)
        self.box_id = t(box_id)
        self.box_params = t(params)
        self.a = torch.tensor([d["a_start"] for d in boxes], dtype=torch.float64, device=dev)
        self.aHdt = torch.zeros((self.n_boxes, 3), dtype=torch.float64, device=dev)
        m = 2 * n - 1
        z = lambda *s, dt=torch.float32: torch.zeros(s, dtype=dt, device=dev)
        self.codes = z(n, dt=torch.uint64)
        self.codes_sorted = z(n, dt=torch.uint64)
        self.perm = z(n, dt=torch.uint32)
        self._alt = [z(n) for _ in range(6)]
        self.child = torch.full((m, 2), -1, dtype=torch.int32, device=dev)
        self.parent = torch.full((m,), -1, dtype=torch.int32, device=dev)
        self.ranges = z(max(n - 1, 1), 2, dt=torch.int32)
        self.counts = z(m, dt=torch.int32)
        self.root_idx = z(1, dt=torch.int32)
        self.n_mass, self.n_com = z(m), z(m, 3)
        self.n_min, self.n_max = z(m, 3), z(m, 3)
        self.table = z(4, m, 4)
        self.workspace = z(4 + 4 * n, dt=torch.int32)
        self.box_roots = z(self.n_boxes, dt=torch.int32)
        self.force = z(n, 3)
        self.stats = z(4, dt=torch.int64)
        self.theta_per_bucket = None
        self.ewald_table = None
        if self.mac == _lib.MAC_EWALD:
            # every box is periodic on its own unit cube: one correction table serves all
            self.ewald_table = z((EWALD_NT + 1) ** 3, 24)
            _lib.call("cnb_ewald_table", self.ewald_table.data_ptr(), EWALD_NT, self._st())
        self._ctx = SortContext(n)
        # full Morton keys below the box bits: the previous step's order mostly holds
        self._ctx.set_mode("adaptive")
        self._graph = None

    # ------------------------------------------------------------ step parts
    def _st(self):
        return int(torch.cuda.current_stream(self.device).cuda_stream)

    def sort_and_build(self):
        """Keys, sort, permutation, tree, node table, buckets and box roots."""
        st = self._st()
        n, m = self.n, 2 * self.n - 1
        p = self.pos
        _lib.call("cnb_compute_codes_boxes", p[0].data_ptr(), p[1].data_ptr(), p[2].data_ptr(),
                  self.box_id.data_ptr(), self.codes.data_ptr(), n, self.box_bits, st)
        self._ctx.sort_pairs(self.codes.data_ptr(), self.codes_sorted.data_ptr(), None,
                             self.perm.data_ptr(), n, 63, st)
        src = self.pos + self.vel
        sa = (C.c_void_p * 6)(*[t.data_ptr() for t in src])
        da = (C.c_void_p * 6)(*[t.data_ptr() for t in self._alt])
        _lib.call("cnb_gather_f32", self.perm.data_ptr(), 6, sa, da, n, st)
        self.pos, self.vel, self._alt = self._alt[:3], self._alt[3:], src
        status = status_buffer(self.device.index).data_ptr()
        _lib.call("cnb_reset_tree_buffers", self.child.data_ptr(), self.parent.data_ptr(),
                  self.counts.data_ptr(), self.root_idx.data_ptr(), m, st)
        _lib.call("cnb_build_tree_ranges", self.codes_sorted.data_ptr(), self.child.data_ptr(),
                  self.parent.data_ptr(), self.ranges.data_ptr(), n, st)
        p = self.pos
        _lib.call("cnb_upward", p[0].data_ptr(), p[1].data_ptr(), p[2].data_ptr(), self.mass.data_ptr(),
                  self.child.data_ptr(), self.parent.data_ptr(), self.n_mass.data_ptr(),
                  self.n_com.data_ptr(), self.n_min.data_ptr(), self.n_max.data_ptr(), None,
                  self.counts.data_ptr(), n, _lib.UPWARD_PLAIN, None, status, st)
        _lib.call("cnb_pack_nodes", self.n_mass.data_ptr(), self.n_com.data_ptr(),
                  self.n_min.data_ptr(), self.n_max.data_ptr(), self.child.data_ptr(),
                  self.table.data_ptr(), m, st)
        _lib.call("cnb_make_buckets_boxes", self.ranges.data_ptr(), self.parent.data_ptr(),
                  self.codes_sorted.data_ptr(), self.box_bits, n, 32 * self.bpl,
                  self.workspace.data_ptr(), st)
        _lib.call("cnb_box_roots", self.ranges.data_ptr(), self.parent.data_ptr(),
                  self.codes_sorted.data_ptr(), self.box_bits, n, self.n_boxes,
                  self.box_roots.data_ptr(), st)

    def compute_forces(self, theta_per_bucket=None, bucket_inter=None):
        """Forces of every box; `bucket_inter` (device int32 per bucket slot,
        periodic law only) receives each bucket's interactions per body."""
        st = self._st()
        tpb = theta_per_bucket if theta_per_bucket is not None else self.theta_per_bucket
        p = self.pos
        if self.ewald_table is not None:
            _lib.call("cnb_forces_grouped_boxes_ewald", p[0].data_ptr(), p[1].data_ptr(),
                      p[2].data_ptr(), self.table.data_ptr(), self.workspace.data_ptr(),
                      self.force.data_ptr(), self.n, self.codes_sorted.data_ptr(), self.box_bits,
                      self.box_roots.data_ptr(), self.box_params.data_ptr(),
                      tpb.data_ptr() if tpb is not None else None, self.bpl, self.block_warps, self.G,
                      self.ewald_table.data_ptr(), EWALD_NT,
                      bucket_inter.data_ptr() if bucket_inter is not None else None,
                      self.stats.data_ptr(), status_buffer(self.device.index).data_ptr(), st)
            return
        _lib.call("cnb_forces_grouped_boxes", p[0].data_ptr(), p[1].data_ptr(), p[2].data_ptr(),
                  self.table.data_ptr(), self.workspace.data_ptr(), self.force.data_ptr(), self.n,
                  self.codes_sorted.data_ptr(), self.box_bits, self.box_roots.data_ptr(),
                  self.box_params.data_ptr(), tpb.data_ptr() if tpb is not None else None, self.mac,
                  self.bpl, self.block_warps, self.G, self.stats.data_ptr(), status_buffer(self.device.index).data_ptr(), st)

    def integrate(self):
        """Per-box Hubble rate and time step on the device, then kick/drift and a += da."""
        a = self.a
        H = self.H0 * torch.sqrt(self.omega_m * a ** -3 + self.omega_l)
        self.aHdt[:, 0] = a
        self.aHdt[:, 1] = H
        self.aHdt[:, 2] = self.da / (a * H) * 0.8
        p, v = self.pos, self.vel
        _lib.call("cnb_integrate_boxes", p[0].data_ptr(), p[1].data_ptr(), p[2].data_ptr(),
                  v[0].data_ptr(), v[1].data_ptr(), v[2].data_ptr(), self.force.data_ptr(),
                  self.codes_sorted.data_ptr(), self.box_bits, self.n, self.aHdt.data_ptr(), self._st())
        self.a += self.da

    def step(self):
        self.sort_and_build()
        self.compute_forces()
        self.integrate()

    # ------------------------------------------------------------ CUDA graph
    def capture(self, warmup=1):
        """Capture one full step in a CUDA graph.  The step alternates between
        two array sets, so two consecutive steps are captured (one replay =
        two steps) and the arrays are back in place after every replay."""
        for _ in range(warmup):
            self.step()
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.step()
            self.step()
        self._graph = g
        return g

    def replay(self):
        """Two steps through the captured graph."""
        self._graph.replay()

    def check(self):
        return check_status(self.device.index)

    # ------------------------------------------------------------ views
    def box_slice(self, b):
        return slice(int(self.offsets[b]), int(self.offsets[b + 1]))

    def n_buckets(self):
        return int(self.workspace[0].item())

    def buckets(self):
        nb = self.n_buckets()
        return self.workspace[4:4 + 4 * nb].view(nb, 4)
