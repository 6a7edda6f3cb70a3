"""Radix-tree manager (src/core/octree.py of the reference), on libcnb.

`OctreeManager(n_bodies, tpb)` allocates the reference's buffers
(octree.py:14-43); `build(pos_d, mass_d, codes_d)` runs reset, Karras build,
upward pass, CoM normalisation and root search (octree.py:45-83) and returns
`root_idx`; `get_buffers()` returns the reference's dict (octree.py:85-93).

Options beyond the reference: `upward="compensated"` (two-sum float32 sums
and a float64 root, `self.root_f64` = [mass, com x, y, z]), and
`node_table=True`, which also builds what the grouped force traversal reads:
the node table (`self.node_table`, [4, M, 4] float32), the node ranges and
the bucket table (`self.workspace`, buckets of at most `bucket` bodies).
With the plain upward pass and buckets of at most 64 bodies the tree is two
launches: the Karras build fused with the ranges, climb counters, root index
and bucket tables (and the super-bucket table of `set_super_table`), then
the bucketed upward pass; the reference-layout arrays are then filled from
the node table when `get_buffers()` asks for them.
"""
from __future__ import annotations

import torch

from .. import _lib
from .._arrays import status_buffer


class OctreeManager:
    """octree.py:13-93."""

    def __init__(self, n_bodies, tpb=256, device=None, upward="plain", node_table=False,
                 bucket=32, quad=False):
        self.n = int(n_bodies)
        self.n_nodes = max(2 * self.n - 1, 1)
        self.tpb = tpb
        self.bpg = (self.n + tpb - 1) // tpb
        dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.device = dev
        m = self.n_nodes
        self.child = torch.full((m, 2), -1, dtype=torch.int32, device=dev)
        self.parent = torch.full((m,), -1, dtype=torch.int32, device=dev)
        self.root_idx = torch.zeros(1, dtype=torch.int32, device=dev)
        self.mass = torch.zeros(m, dtype=torch.float32, device=dev)
        self.com = torch.zeros((m, 3), dtype=torch.float32, device=dev)
        self.aabb_min = torch.zeros((m, 3), dtype=torch.float32, device=dev)
        self.aabb_max = torch.zeros((m, 3), dtype=torch.float32, device=dev)
        self.counters = torch.zeros(m, dtype=torch.int32, device=dev)
        if upward not in ("plain", "compensated"):
            raise ValueError("upward must be 'plain' or 'compensated'")
        self.upward = upward
        self.err = torch.zeros((m, 4), dtype=torch.float32, device=dev) if upward == "compensated" else None
        self.root_f64 = torch.zeros(4, dtype=torch.float64, device=dev)
        # True after the fused pass: the reference-layout arrays are filled on demand
        self._stale_ref = False
        self.node_table = None
        if node_table:
            # traversal records and boxes, node ranges and the bucket table
            self.node_table = torch.empty((4, m, 4), dtype=torch.float32, device=dev)
            self.sums = torch.empty((m, 4), dtype=torch.float32, device=dev)   # climb scratch
            self.ranges = torch.zeros((max(self.n - 1, 1), 2), dtype=torch.int32, device=dev)
            self.workspace = torch.zeros(4 + 4 * max(self.n, 1), dtype=torch.int32, device=dev)
            self.bucket = int(bucket)
        # second central moments of the internal nodes (grouped plain upward only)
        self.quad = torch.zeros((m, 8), dtype=torch.float32, device=dev) if quad else None
        if quad and (not node_table or upward != "plain"):
            raise ValueError("quad needs node_table=True and the plain upward pass")
        self.super_ws, self.super_bodies = None, 0
        self._super_built = None

    def _stream(self):
        return int(torch.cuda.current_stream(self.device).cuda_stream)

    def set_super_table(self, super_ws, super_bodies):
        """Also build the super-bucket table (super-buckets of at most
        `super_bodies` bodies) into `super_ws` with every tree, for the
        two-level walk; (None, 0) stops it."""
        self.super_ws = super_ws
        self.super_bodies = int(super_bodies) if super_ws is not None else 0
        self._super_built = None   # made by the next build

    @property
    def _fused_build(self):
        # tree, buckets and root in one launch, then the bucketed upward pass
        return self.node_table is not None and self.upward == "plain" and self.bucket <= 64

    @property
    def super_table_current(self):
        """True when `super_ws` holds the super-bucket table of the current tree
        for the current `super_bodies` (made by the last build)."""
        return (self.super_ws is not None and
                self._super_built == (self.super_ws.data_ptr(), self.super_bodies))

    def build(self, pos_d, mass_d, codes_d):
        """octree.py:45-83: reset, build_tree, compute_multipoles, normalize_com, find_root."""
        st = self._stream()
        n, m = self.n, self.n_nodes
        status = status_buffer(self.device.index).data_ptr()
        px, py, pz = pos_d
        if self._fused_build:
            # one launch builds the tree, its ranges, the bucket tables and the root index
            # and zeroes the climb counters (leaf children and the root's parent keep the -1
            # they were allocated with); then sums, boxes and the traversal table bucket by
            # bucket and above the buckets; com stays raw
            _lib.call("cnb_build_tree_buckets", codes_d.data_ptr(), self.child.data_ptr(),
                      self.parent.data_ptr(), self.ranges.data_ptr(), self.counters.data_ptr(),
                      self.root_idx.data_ptr(), n, self.bucket, self.workspace.data_ptr(),
                      self.super_bodies, self.super_ws.data_ptr() if self.super_ws is not None else None,
                      st)
            _lib.call("cnb_upward_table_buckets", px.data_ptr(), py.data_ptr(), pz.data_ptr(),
                      mass_d.data_ptr(), self.child.data_ptr(), self.parent.data_ptr(),
                      self.workspace.data_ptr(), self.counters.data_ptr(),
                      self.node_table.data_ptr(), self.sums.data_ptr(),
                      self.quad.data_ptr() if self.quad is not None else None, n, status, st)
            self._stale_ref = True
            self._super_built = ((self.super_ws.data_ptr(), self.super_bodies)
                                 if self.super_ws is not None else None)
            return self.root_idx
        self._super_built = None
        _lib.call("cnb_reset_tree_buffers", self.child.data_ptr(), self.parent.data_ptr(),
                  self.counters.data_ptr(), self.root_idx.data_ptr(), m, st)
        if self.node_table is not None:
            _lib.call("cnb_build_tree_ranges", codes_d.data_ptr(), self.child.data_ptr(),
                      self.parent.data_ptr(), self.ranges.data_ptr(), n, st)
        else:
            _lib.call("cnb_build_tree", codes_d.data_ptr(), self.child.data_ptr(), self.parent.data_ptr(), n, st)
        if self.node_table is not None and self.upward == "plain":
            # one pass: sums, boxes and the traversal table; com stays raw until asked for
            if self.quad is not None:
                _lib.call("cnb_upward_table_quad", px.data_ptr(), py.data_ptr(), pz.data_ptr(),
                          mass_d.data_ptr(), self.child.data_ptr(), self.parent.data_ptr(),
                          self.counters.data_ptr(), self.node_table.data_ptr(),
                          self.sums.data_ptr(), self.quad.data_ptr(), n, status, st)
            else:
                _lib.call("cnb_upward_table", px.data_ptr(), py.data_ptr(), pz.data_ptr(),
                          mass_d.data_ptr(), self.child.data_ptr(), self.parent.data_ptr(),
                          self.counters.data_ptr(), self.node_table.data_ptr(), self.sums.data_ptr(),
                          n, status, st)
            self._stale_ref = True
            _lib.call("cnb_find_root", self.parent.data_ptr(), self.root_idx.data_ptr(), m, st)
            _lib.call("cnb_make_buckets", self.ranges.data_ptr(), self.parent.data_ptr(), n,
                      self.bucket, self.workspace.data_ptr(), st)
            return self.root_idx
        mode = _lib.UPWARD_COMPENSATED if self.upward == "compensated" else _lib.UPWARD_PLAIN
        _lib.call("cnb_upward", px.data_ptr(), py.data_ptr(), pz.data_ptr(), mass_d.data_ptr(),
                  self.child.data_ptr(), self.parent.data_ptr(), self.mass.data_ptr(),
                  self.com.data_ptr(), self.aabb_min.data_ptr(), self.aabb_max.data_ptr(),
                  self.err.data_ptr() if self.err is not None else None, self.counters.data_ptr(), n,
                  mode, self.root_f64.data_ptr() if self.err is not None else None, status, st)
        _lib.call("cnb_find_root", self.parent.data_ptr(), self.root_idx.data_ptr(), m, st)
        if self.node_table is not None:
            _lib.call("cnb_pack_nodes", self.mass.data_ptr(), self.com.data_ptr(),
                      self.aabb_min.data_ptr(), self.aabb_max.data_ptr(), self.child.data_ptr(),
                      self.node_table.data_ptr(), m, st)
            _lib.call("cnb_make_buckets", self.ranges.data_ptr(), self.parent.data_ptr(), n,
                      self.bucket, self.workspace.data_ptr(), st)
        return self.root_idx

    def validate(self):
        """Check the topology of the current tree (raises CnbError if invalid)."""
        from .._arrays import check_status
        scratch = torch.empty(2 * max(self.n, 1), dtype=torch.int32, device=self.device)
        _lib.call("cnb_validate_tree", self.child.data_ptr(), self.parent.data_ptr(), self.n,
                  scratch.data_ptr(), status_buffer(self.device.index).data_ptr(), self._stream())
        return check_status(self.device.index)

    def rebucket(self, max_size):
        """Rebuild the bucket table of the current tree with buckets of at most max_size bodies."""
        self.bucket = int(max_size)
        if self.node_table is not None and self.n > 0:
            st = self._stream()
            _lib.call("cnb_make_buckets", self.ranges.data_ptr(), self.parent.data_ptr(), self.n,
                      self.bucket, self.workspace.data_ptr(), st)

    def get_buffers(self):
        """octree.py:85-93 (filled from the node table if the fused pass built the tree)."""
        if self._stale_ref:
            _lib.call("cnb_unpack_nodes", self.node_table.data_ptr(), self.mass.data_ptr(),
                      self.com.data_ptr(), self.aabb_min.data_ptr(), self.aabb_max.data_ptr(),
                      self.n_nodes, self._stream())
            self._stale_ref = False
        return {
            "child": self.child,
            "mass": self.mass,
            "com": self.com,
            "min": self.aabb_min,
            "max": self.aabb_max,
            "root": self.root_idx,
        }
