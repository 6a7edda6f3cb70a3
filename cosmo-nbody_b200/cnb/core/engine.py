"""Simulation engine (src/core/engine.py of the reference), on libcnb.

`SimulationEngine(config, state)` with `step()` and `run()` keeps the
reference's sequence (engine.py:55-123): Hubble rate and time step on the
host, Morton sort, tree build, forces, kick/drift, `a += da`.  Differences:
the forces are one launch over all bodies (the reference launches 5 000
bodies at a time), the step does not synchronise the device, and the force
kernel is chosen by config.FORCE_MODE:

  "reference"  per-particle stack traversal with the reference's opening
               test (config.PRECISION "f64" = the reference's arithmetic,
               "f32" = float32);
  "grouped"    warp-per-bucket traversal (config.MAC "ref_x": the reference's
               opening decisions body by body, so every body gets the
               reference's node set; "ref_x_bucket": the reference's test
               decided once per bucket, finer node sets; "periodic";
               "ewald" = the periodic force law, not the reference's minimum
               image; optional per-bucket theta from `theta_per_group`); with
               config.SUPER_BODIES > 0 and a reference test, the two-level
               form (super-buckets of that many bodies walk the top of the
               tree once for all their buckets).

Device error flags are read by `check()` (one synchronisation).
"""
from __future__ import annotations

import torch

from .. import _lib
from .._arrays import check_status, status_buffer
from ..utils.cosmology import get_hubble_param
from .camera import Camera
from .octree import OctreeManager

MACS = {"ref_x": _lib.MAC_REF_X, "ref_x_bucket": _lib.MAC_REF_X_BUCKET,
        "periodic": _lib.MAC_PERIODIC, "ewald": _lib.MAC_EWALD}
EWALD_NT = 64   # Ewald correction table: 65^3 points on [0, 1/2]^3


class SimulationEngine:
    def __init__(self, config, state, camera=True):
        self.config = config
        self.state = state
        self.force_mode = getattr(config, "FORCE_MODE", "reference")
        if self.force_mode not in ("reference", "grouped"):
            raise ValueError("FORCE_MODE must be 'reference' or 'grouped'")
        self.bodies_per_lane = int(getattr(config, "BODIES_PER_LANE", 1))
        self.block_warps = int(getattr(config, "BLOCK_WARPS", 8))
        self.quadrupole = bool(getattr(config, "QUADRUPOLE", False))
        if self.quadrupole and getattr(config, "MAC", "ref_x") != "ewald":
            raise ValueError("QUADRUPOLE needs MAC 'ewald'")
        self.tree_manager = OctreeManager(state.n, config.TPB, device=state.device,
                                          upward=getattr(config, "UPWARD", "plain"),
                                          node_table=self.force_mode == "grouped",
                                          bucket=32 * self.bodies_per_lane, quad=self.quadrupole)
        res = getattr(config, "RES", 1024)
        self.camera = Camera(config.N_STEPS, res, config, device=state.device) if camera else None
        self.cache_size = getattr(config, "CACHE_SIZE", 256)
        self.tpb = config.TPB
        self.a = config.A_START
        self.da = (config.A_END - config.A_START) / config.N_STEPS
        self.top_nodes = torch.full((self.cache_size,), -1, dtype=torch.int32, device=state.device)
        self.node_to_cache = torch.full((self.tree_manager.n_nodes,), -1, dtype=torch.int32,
                                        device=state.device)
        self.theta_per_group = None   # float32 per bucket slot (device), grouped mode only
        # learned opening-angle controller (cnb.controller.ThetaController); None = plain theta
        self.controller = None
        self.controller_scale = 1.0
        # periodic law: device int32 per bucket slot receiving each bucket's
        # interactions per body (None: not recorded)
        self.bucket_inter = None
        # the controller's acceleration input: None = the previous step's forces
        # (state.force); a tensor [N, 3] in the current sorted order overrides it
        self.controller_accel = None
        self._bucket_order = None
        # True while state.force holds forces in the current sorted order (a
        # sort since the last force stage leaves it in the previous order)
        self._force_current = False
        self.stats = torch.zeros(4, dtype=torch.int64, device=state.device)
        self.mac = MACS[getattr(config, "MAC", "ref_x")]
        # periodic test: image-ambiguous nodes of at most SLAB_BODIES bodies' mass are applied
        # with the per-pair minimum image (0 = exact)
        self.slab_mass = float(getattr(config, "SLAB_BODIES", 0)) / max(state.n, 1)
        self.ewald_table = None
        if self.mac == _lib.MAC_EWALD:
            if self.force_mode != "grouped":
                raise ValueError("MAC 'ewald' needs FORCE_MODE 'grouped'")
            self.ewald_table = torch.empty(((EWALD_NT + 1) ** 3, 24), dtype=torch.float32,
                                           device=state.device)
            _lib.call("cnb_ewald_table", self.ewald_table.data_ptr(), EWALD_NT, self._stream())
        self.super_bodies = 0
        self.super_ws = None
        if self.force_mode == "grouped":
            self.set_super_bodies(int(getattr(config, "SUPER_BODIES", 0)))
        self.precision = _lib.PREC_F64 if getattr(config, "PRECISION", "f32") == "f64" else _lib.PREC_F32
        self.stage_events = None
        self.nvtx = False          # NVTX ranges around the step's stages (for nsys / ncu timelines)
        self._nvtx_open = False

    def set_super_bodies(self, super_bodies):
        """Two-level walk with super-buckets of at most `super_bodies` bodies
        (0: single level).  Needs the grouped mode and the reference's test
        ("ref_x" or "ref_x_bucket")."""
        super_bodies = int(super_bodies)
        if super_bodies == 0:
            self.super_bodies, self.super_ws = 0, None
            self.tree_manager.set_super_table(None, 0)
            return
        if self.force_mode != "grouped" or self.mac not in (_lib.MAC_REF_X, _lib.MAC_REF_X_BUCKET):
            raise ValueError("SUPER_BODIES needs FORCE_MODE 'grouped' and MAC 'ref_x' or 'ref_x_bucket'")
        nbytes = int(_lib.load().cnb_two_level_workspace_bytes(self.state.n, super_bodies))
        if nbytes < 0:
            raise ValueError("SUPER_BODIES must be at least 32")
        if self.super_ws is None or self.super_ws.numel() * 4 < nbytes:
            self.super_ws = torch.empty((nbytes + 15) // 16, 4, dtype=torch.int32,
                                        device=self.state.device)
        self.super_bodies = super_bodies
        # the tree build makes the super-bucket table too
        self.tree_manager.set_super_table(self.super_ws, super_bodies)

    def _stream(self):
        return int(torch.cuda.current_stream(self.state.device).cuda_stream)

    def compute_forces(self):
        """The force stage of engine.py:91-111, one launch over all bodies."""
        self._compute_forces()
        self._force_current = True

    def _compute_forces(self):
        cfg, s, tm = self.config, self.state, self.tree_manager
        st = self._stream()
        status = status_buffer(s.device.index).data_ptr()
        px, py, pz = s.pos
        if self.force_mode == "grouped":
            if self.controller is not None:
                # learned per-bucket theta (fused features + network on the GPU)
                # the previous step's accelerations, row s.perm[i] for the body now at i
                if self.controller_accel is not None:
                    accel, perm = self.controller_accel, None
                else:
                    accel, perm = s.force, (None if self._force_current else s.perm)
                self.theta_per_group = self.controller.theta_for_buckets(
                    tm.node_table, tm.parent, tm.workspace, s.n, accel, perm,
                    out=self.theta_per_group, scale=self.controller_scale)
            tpg = self.theta_per_group
            order = None
            if self.ewald_table is not None and tpg is not None:
                # per-bucket angles: the most expensive buckets are handed out first
                if self._bucket_order is None or self._bucket_order.numel() < tpg.numel():
                    self._bucket_order = torch.empty(tpg.numel(), dtype=torch.int32, device=s.device)
                order = self._bucket_order
                _lib.call("cnb_order_buckets", tpg.data_ptr(), tm.workspace.data_ptr(),
                          order.data_ptr(), st)
            if self.ewald_table is not None:
                _lib.call("cnb_forces_grouped_ewald", px.data_ptr(), py.data_ptr(), pz.data_ptr(),
                          tm.node_table.data_ptr(), tm.workspace.data_ptr(), s.force.data_ptr(), s.n,
                          float(cfg.THETA), tpg.data_ptr() if tpg is not None else None,
                          self.bodies_per_lane, self.block_warps, float(cfg.G), float(cfg.SOFTENING),
                          self.ewald_table.data_ptr(), EWALD_NT,
                          tm.quad.data_ptr() if tm.quad is not None else None,
                          order.data_ptr() if order is not None else None,
                          self.bucket_inter.data_ptr() if self.bucket_inter is not None else None,
                          self.stats.data_ptr(), status, st)
                return
            if self.super_ws is not None and tpg is None:
                # NULL ranges and parents: the super-bucket table was built with the tree
                # (otherwise, e.g. after a change of super_bodies, the call builds it)
                built = tm.super_table_current
                _lib.call("cnb_forces_two_level", px.data_ptr(), py.data_ptr(), pz.data_ptr(),
                          tm.node_table.data_ptr(), None if built else tm.ranges.data_ptr(),
                          None if built else tm.parent.data_ptr(),
                          tm.workspace.data_ptr(), self.super_ws.data_ptr(),
                          self.super_ws.numel() * 4, self.super_bodies, s.force.data_ptr(), s.n,
                          float(cfg.THETA), self.mac, self.bodies_per_lane, self.block_warps, float(cfg.G),
                          float(cfg.SOFTENING), float(cfg.BOX_SIZE), self.stats.data_ptr(), status, st)
                return
            _lib.call("cnb_forces_grouped", px.data_ptr(), py.data_ptr(), pz.data_ptr(),
                      tm.node_table.data_ptr(), tm.workspace.data_ptr(), s.force.data_ptr(), s.n,
                      float(cfg.THETA), tpg.data_ptr() if tpg is not None else None, self.mac,
                      self.bodies_per_lane, self.block_warps, float(cfg.G), float(cfg.SOFTENING),
                      float(cfg.BOX_SIZE), self.slab_mass, self.stats.data_ptr(), status, st)
        else:
            _lib.call("cnb_compute_forces", px.data_ptr(), py.data_ptr(), pz.data_ptr(),
                      tm.child.data_ptr(), tm.mass.data_ptr(), tm.com.data_ptr(),
                      tm.aabb_min.data_ptr(), tm.aabb_max.data_ptr(), s.force.data_ptr(),
                      float(cfg.THETA), float(cfg.G), float(cfg.SOFTENING), float(cfg.BOX_SIZE),
                      tm.root_idx.data_ptr(), 0, s.n, s.n, self.precision, status, st)

    _NEXT_STAGE = {"start": "sort", "sort": "tree", "tree": "forces"}

    def _mark(self, name):
        if self.stage_events is not None:
            ev = torch.cuda.Event(enable_timing=True)
            ev.record()
            self.stage_events.append((name, ev))
        if self.nvtx:
            # a mark ends the stage named after it and opens the next one
            if self._nvtx_open:
                torch.cuda.nvtx.range_pop()
                self._nvtx_open = False
            nxt = self._NEXT_STAGE.get(name)
            if nxt is not None:
                torch.cuda.nvtx.range_push(nxt)
                self._nvtx_open = True

    def forces_only(self):
        """Sort, tree and forces for the current state (no integration)."""
        self._mark("start")
        self.state.sort_buffer_by_morton(self.config)
        self._force_current = False
        self._mark("sort")
        self.tree_manager.build(self.state.pos, self.state.mass, self.state.codes)
        self._mark("tree")
        self.compute_forces()
        self._mark("forces")

    def step(self):
        """engine.py:55-123."""
        H = get_hubble_param(self.a, self.config)
        dt_physics = self.da / (self.a * H) * 0.8
        self.forces_only()
        if self.nvtx:
            torch.cuda.nvtx.range_push("integrate")
            self._nvtx_open = True
        s = self.state
        _lib.call("cnb_integrate", *(t.data_ptr() for t in s.pos + s.vel), s.force.data_ptr(), s.n,
                  float(self.a), float(H), float(dt_physics), self._stream())
        self._mark("integrate")
        self.a += self.da

    # ------------------------------------------------------------ CUDA graph
    def _step_device(self, mvp=None, frame=None):
        """One step with no host scalars (a, H, dt live on the device), so it
        can be captured; `mvp` (device [4,4]) also splats the new positions
        and `frame` (device [H, W, 3]) receives their colourised grid."""
        self.forces_only()
        a = self.a_dev
        cfg = self.config
        H = cfg.H0 * torch.sqrt(cfg.OMEGA_M * a ** -3 + cfg.OMEGA_L)
        self.aHdt[:, 0] = a
        self.aHdt[:, 1] = H
        self.aHdt[:, 2] = self.da / (a * H) * 0.8
        s = self.state
        _lib.call("cnb_integrate_boxes", *(t.data_ptr() for t in s.pos + s.vel), s.force.data_ptr(),
                  s.codes.data_ptr(), 0, s.n, self.aHdt.data_ptr(), self._stream())
        self.a_dev += self.da
        if mvp is not None and self.camera is not None:
            self.camera.splat_device(mvp, *s.pos)
            if frame is not None:
                self.camera.colorize(out=frame)

    def capture(self, splat=True, colorize=False, step0=0):
        """Capture two consecutive steps (and their splats) in one CUDA graph;
        each splat overlaps the step after it.
        The step alternates between two array sets, so after every replay the
        arrays are back where they were captured.  The two steps that run
        eagerly first (steps step0, step0 + 1 of the camera orbit) warm up
        the capture.  With `colorize`, each step's frame lands in
        `frame_slots[k]`.  Use replay() afterwards."""
        dev = self.state.device
        self.a_dev = torch.tensor([self.a], dtype=torch.float64, device=dev)
        self.aHdt = torch.zeros((1, 3), dtype=torch.float64, device=dev)
        self.mvp_slots = torch.zeros((2, 4, 4), dtype=torch.float32, device=dev)
        self._graph_splat = bool(splat and self.camera is not None)
        self.frame_slots = None
        if self._graph_splat:
            for k in range(2):
                self.mvp_slots[k].copy_(self.camera.mvp_host(step0 + k))
            if colorize:
                self.frame_slots = torch.empty((2, self.camera.height, self.camera.width, 3),
                                               dtype=torch.float32, device=dev)

        side = torch.cuda.Stream(dev)

        def two_steps():
            main = torch.cuda.current_stream(dev)
            for k in range(2):
                self._step_device()
                if self._graph_splat:
                    # the splat reads only this step's positions, which the next
                    # step's sort gathers from but does not overwrite: it runs
                    # on a second stream beside that step
                    side.wait_stream(main)
                    with torch.cuda.stream(side):
                        self.camera.splat_device(self.mvp_slots[k], *self.state.pos)
                        if self.frame_slots is not None:
                            self.camera.colorize(out=self.frame_slots[k])
            if self._graph_splat:
                main.wait_stream(side)

        two_steps()                      # warm-up, eager
        self.a += 2 * self.da
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            two_steps()
        self._graph = g
        self._graph_step = step0 + 2
        return g

    def replay(self):
        """Two steps through the captured graph (camera orbit continues)."""
        if self._graph_splat:
            for k in range(2):
                self.mvp_slots[k].copy_(self.camera.mvp_host(self._graph_step + k), non_blocking=True)
        self._graph.replay()
        self._graph_step += 2
        self.a += 2 * self.da

    def save_state(self, path):
        """Checkpoint: positions, velocities, masses, the scale factor and
        the camera step, as one torch file (resume with load_state)."""
        s = self.state
        torch.save({"n": s.n, "pos": [p.cpu() for p in s.pos], "vel": [v.cpu() for v in s.vel],
                    "mass": s.mass.cpu(), "a": float(self.a),
                    "graph_step": int(getattr(self, "_graph_step", 0))}, path)

    def load_state(self, path):
        """Resume from save_state: the arrays are copied into this engine's
        buffers (the body count must match)."""
        d = torch.load(path)
        s = self.state
        if int(d["n"]) != s.n:
            raise ValueError(f"checkpoint has {d['n']} bodies, the engine {s.n}")
        for dst, src in zip(s.pos + s.vel, d["pos"] + d["vel"]):
            dst.copy_(src)
        s.mass.copy_(d["mass"])
        self.a = float(d["a"])
        self._graph = None    # a captured graph holds the old scalars

    def enable_stage_timing(self, on=True):
        """Record CUDA events between the stages of every step (stage_times() reads them)."""
        self.stage_events = [] if on else None

    def stage_times(self):
        """Milliseconds per stage summed over the recorded steps; clears the record."""
        out = {}
        ev = self.stage_events or []
        torch.cuda.synchronize()
        for (a, ea), (b, eb) in zip(ev, ev[1:]):
            if b == "start":
                continue
            out[b] = out.get(b, 0.0) + ea.elapsed_time(eb)
        if self.stage_events is not None:
            self.stage_events = []
        return out

    def run(self, n_steps=None, frames=False, graph=None):
        """engine.py:125-139 without the host video buffer: steps, captures a
        frame per step, returns the last frame (or all frames if `frames`).
        With `graph` (default: grouped mode and at least 4 steps) the steps
        run as replays of one captured two-step graph, frames included, with
        no host synchronisation between them; an odd last step runs eagerly."""
        n_steps = self.config.N_STEPS if n_steps is None else n_steps
        if graph is None:
            graph = self.force_mode == "grouped" and n_steps >= 4
        out = []
        frame = None
        i = 0
        if graph and n_steps >= 2:
            self.capture(splat=True, colorize=True, step0=0)     # runs steps 0 and 1
            i = 2
            while True:
                if self.frame_slots is not None:
                    frame = self.frame_slots[1]
                    if frames:
                        out.extend(f.clone() for f in self.frame_slots)
                if i + 2 > n_steps:
                    break
                self.replay()
                i += 2
            self._graph = None
            if i < n_steps:
                # the device scalars carry a, so the odd last step takes them too
                self._step_device()
                self.a += self.da
                i += 1
                if self.camera is not None:
                    frame = self.camera.capture(i - 1, *self.state.pos)
                    if frames:
                        out.append(frame.clone())
        for i in range(i, n_steps):
            self.step()
            if self.camera is not None:
                frame = self.camera.capture(i, *self.state.pos)
                if frames:
                    out.append(frame.clone())
        self.check()
        return out if frames else frame

    def check(self):
        """Synchronise and raise CnbError if a kernel flagged an error."""
        return check_status(self.state.device.index)
