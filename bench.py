"""Barnes-Hut step benchmark: particle-steps/s at N = 128^3 on one B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (the reference's full plain step at reference scale): 128^3 = 2,097,152
float32 bodies from seeded Zel'dovich initial conditions (seed 1; P(k) ~ k^-2.5,
sigma_disp = 0.3/128, a0 = 0.02, H0 = 67.8, Omega_m = 1, Omega_L = 0.692),
theta = 0.5, softening 0.5/128, G = 1, kick-drift steps of da = 0.002, and the
density splat to a 1920x1080 float32 grid with the orbiting 60-degree camera.
One bench step = one simulation step (63-bit Morton keys, stable sort +
permute, Karras build, upward pass, force traversal, kick/drift) plus the splat.
The force traversal is the reference's (physics_kernels.py:14-153) with its
opening test decided body by body (--mac ref_x): every body gets exactly the
reference's node set.  The line's "variants" entry times the same loop with
the test decided once per 64-body bucket (ref_x_bucket: finer node sets, more
accurate than the reference, not its forces).
The sort is adaptive (--sort auto): the keys of bodies sorted one step earlier
mostly keep their order, so a near-sorted path (take out the keys that break the
order, sort them, merge them back) replaces the full radix sort whenever at most
2048 keys are out of place; both give the same stable argsort, and the line's
"sort" entry counts which one ran.  --sort full times the radix sort every step.

`--impl ours` (default) runs libcnb on the GPU; `--impl reference` times the
reference's algorithm (the CPU oracle restating src/kernels/*.py, all host
threads) on the same workload, every stage on every body (about 3.5 s per
step on 16 cores; --cpu-sample K times the force traversal on K targets and
scales it instead).  `--impl reference-gpu` launches the reference's own
Numba kernels on the GPU (run_reference_gpu).  Under torchrun each rank runs
an independent box (seed 1 + 1000 * rank: replicas, weak scaling); rank 0
prints the JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "cosmo-nbody_b200"))

METRIC = "particle-steps/s at N=128^3 (full plain step + 1920x1080 splat)"


def metric_for(n_grid):
    """The metric string for an n_grid^3 run (METRIC for the default 128^3)."""
    return METRIC.replace("N=128^3", f"N={n_grid}^3")
N_GRID = 128
FLOPS_PER_INTERACTION = 20   # 3 sub, 3 min-image, 5 d2, 1 +eps2, 1 rsqrt, 3 mul, 3 fma (+1)
FULL_SORT_KERNELS = 10     # zeroing + digit histogram + 8 one-sweep passes (63-bit keys)
E2E_MIN_STEPS = 40         # steps of the end-to-end measurement (at least --steps)
# DRAM traffic (dram__bytes_read.sum + dram__bytes_write.sum) of one force-kernel launch on
# the 128^3 seed-1 workload at theta 0.5 (64-body buckets, two-level walk with 512-body
# super-buckets), from one ncu capture of each kernel; not measured by this run
FORCES_TRAFFIC_BYTES_128 = {"ref_x": 202.8e6 + 21.2e6, "ref_x_bucket": 213.2e6 + 21.8e6}
FORCES_KERNEL = {"ref_x": "k_forces_exact", "ref_x_bucket": "k_forces_grouped",
                 "periodic": "k_forces_grouped", "ewald": "k_forces_grouped"}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference", "reference-gpu"])
    ap.add_argument("--n-grid", type=int, default=N_GRID)
    ap.add_argument("--theta", type=float, default=0.5)
    ap.add_argument("--force-mode", default="grouped", choices=["grouped", "reference"])
    ap.add_argument("--mac", default="ref_x", choices=["ref_x", "ref_x_bucket", "periodic", "ewald"],
                    help="opening test; 'ewald' also switches to the periodic force law")
    ap.add_argument("--precision", default="f32", choices=["f32", "f64"],
                    help="arithmetic of the reference force mode (f64 = the reference's)")
    ap.add_argument("--upward", default="plain", choices=["plain", "compensated"])
    ap.add_argument("--bpl", type=int, default=1, choices=[1, 2], help="bodies per lane (grouped)")
    ap.add_argument("--warps", type=int, default=8, choices=[2, 4, 8],
                    help="warps per block of the grouped traversal (with --no-tune)")
    ap.add_argument("--slab", type=float, default=0, help="periodic test: slab tolerance in bodies")
    ap.add_argument("--sort", default="auto", choices=["auto", "full", "adaptive"],
                    help="sort: auto = near-sorted path first (morton63 keys), full = radix sort every step")
    ap.add_argument("--quad", action="store_true",
                    help="with --mac ewald: internal nodes also apply their quadrupole moments")
    ap.add_argument("--super", type=int, default=0,
                    help="super-bucket size of the two-level walk (ref_x test; 0 = single level)")
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--accuracy-sample", type=int, default=4096)
    ap.add_argument("--cpu-sample", type=int, default=0,
                    help="reference arm: force traversal on this many evenly spaced targets scaled "
                         "to N (0: every body, no extrapolation)")
    ap.add_argument("--no-graph", dest="graph", action="store_false",
                    help="launch every kernel from Python instead of replaying a CUDA graph")
    ap.add_argument("--no-tune", action="store_true", help="skip the launch-shape autotuner")
    ap.add_argument("--no-learned", dest="learned", action="store_false",
                    help="skip the learned-theta against plain-theta comparison")
    ap.add_argument("--learned-sample", type=int, default=4096,
                    help="float64 periodic direct-sum sample of the learned-theta comparison")
    ap.add_argument("--profile", action="store_true",
                    help="timed loop only (no e2e, accuracy, CPU baseline or clock sampling)")
    return ap.parse_args()


def make_config(args, seed):
    from cnb.utils import config as cfgmod
    n = args.n_grid
    return cfgmod.make(N_GRID=n, SOFTENING=0.5 / n, THETA=args.theta, N_STEPS=10,
                       A_START=0.02, A_END=0.02 + 10 * 0.002, KEY_MODE="morton63",
                       FORCE_MODE=args.force_mode, MAC=args.mac, PRECISION=args.precision,
                       UPWARD=args.upward, RES=args.width, RES_W=args.width, RES_H=args.height,
                       SEED=seed, BODIES_PER_LANE=args.bpl, SLAB_BODIES=args.slab,
                       SUPER_BODIES=args.super, BLOCK_WARPS=args.warps, QUADRUPOLE=args.quad,
                       SORT_MODE=args.sort)


def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return ws, rank, local


def replica_seed(rank):
    """Seed of the independent box a rank simulates (replicas, weak scaling)."""
    return 1 + 1000 * rank


def max_over_ranks(x, ws, device="cuda"):
    """The largest value of x over all ranks (the job's time is its slowest rank's)."""
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(bodies_per_rank, steps, ws, max_ms):
    """Whole-job particle-steps/s: every rank's bodies x steps over the slowest rank's time."""
    return ws * bodies_per_rank * steps / (max_ms * 1e-3)


def barrier(ws):
    import torch
    torch.cuda.synchronize()
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 200 ms."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if self.proc is None or not self.path:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}

        def num(s):
            try:
                return float(s)
            except ValueError:
                return None
        sm = [num(r[1]) for r in rows if num(r[1]) is not None]
        mx = [num(r[2]) for r in rows if num(r[2]) is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return {"hbm_gbs": d.get("hbm_gbs", 6650.0), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def fma_peak_tflops(detail=None):
    """Measured FP32 FMA throughput (libcnb probes), TFLOP/s: the higher of
    scalar FFMA chains and packed FFMA2 chains (the force loops issue FFMA2).
    detail (dict, optional) receives both figures."""
    import torch
    from cnb import _lib
    blocks = 148 * 16
    out = torch.empty(blocks * 256, dtype=torch.float32, device="cuda")
    iters = 20000
    st = int(torch.cuda.current_stream().cuda_stream)
    res = {}
    for name, flops_per_iter in (("cnb_fma_probe", 16.0), ("cnb_fma2_probe", 32.0)):
        for _ in range(2):
            _lib.call(name, out.data_ptr(), iters, blocks, st)
        best = 0.0
        for _ in range(3):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            _lib.call(name, out.data_ptr(), iters, blocks, st)
            e1.record()
            e1.synchronize()
            ms = e0.elapsed_time(e1)
            best = max(best, flops_per_iter * iters * blocks * 256 / (ms * 1e-3) / 1e12)
        res["ffma" if name == "cnb_fma_probe" else "ffma2"] = best
    if detail is not None:
        detail.update(res)
    return max(res.values())


# ---------------------------------------------------------------- CPU (reference algorithm)

def cpu_reference_step(pos, vel, mass, a, da, cfg, sample, threads, full_check=False):
    """One step of the reference's algorithm on the host (oracle restating
    src/core/engine.py:55-123 with the 63-bit key), forces on `sample`
    evenly spaced targets scaled to N.  Returns (new pos, new vel, seconds);
    with `full_check` also a dict comparing the scaled sample with the force
    traversal timed on every body of the same tree."""
    from oracle import oracle as orc
    n = pos[0].size
    t0 = time.perf_counter()
    H = orc.hubble(a)
    dt = da / (a * H) * 0.8
    spos, svel, smass, codes, _ = orc.sort_state(pos, vel, mass, orc.KEY_MORTON63)
    ch, par = orc.build_tree(codes)
    nm, nc, lo, hi = orc.compute_multipoles(*spos, smass, ch, par)
    root = orc.find_root(par)
    t1 = time.perf_counter()
    targets = (np.linspace(0, n - 1, min(sample, n)).astype(np.int64) if sample > 0
               else np.arange(n, dtype=np.int64))
    orc.forces_targets_f64(*spos, ch, nm, nc, lo, hi, cfg.THETA, cfg.G, cfg.SOFTENING,
                           cfg.BOX_SIZE, root, targets, nthreads=threads)
    t2 = time.perf_counter()
    force = np.zeros((n, 3), np.float32)  # untimed stand-in for the unsampled targets
    t3 = time.perf_counter()
    new = orc.integrate(*spos, *svel, force, a, H, dt)
    from cnb.utils.visualizer import get_mvp_matrix
    mvp = get_mvp_matrix(0, (0.5, 0.5, 0.5), 1.0, cfg, aspect=cfg.RES_W / cfg.RES_H)
    orc.render_density(*new[:3], mvp, cfg.RES_W, cfg.RES_H)
    t4 = time.perf_counter()
    seconds = (t1 - t0) + (t2 - t1) * n / targets.size + (t4 - t3)
    if not full_check:
        return new[:3], new[3:], seconds
    t5 = time.perf_counter()
    orc.forces_targets_f64(*spos, ch, nm, nc, lo, hi, cfg.THETA, cfg.G, cfg.SOFTENING,
                           cfg.BOX_SIZE, root, np.arange(n, dtype=np.int64), nthreads=threads)
    full = time.perf_counter() - t5
    scaled = (t2 - t1) * n / targets.size
    check = {"force_targets_sampled": int(targets.size), "force_s_scaled_from_sample": scaled,
             "force_s_all_bodies_timed": full, "timed_over_scaled": full / scaled}
    return new[:3], new[3:], seconds, check


def _sample_text(sample, n):
    if 0 < sample < n:
        return (f"all stages on all {n} bodies; force traversal (reference per-body algorithm, "
                f"float64) on {sample} evenly spaced targets scaled to N")
    return f"one full step: every stage, force traversal (float64) on all {n} bodies"


def run_reference(args):
    ws, rank, _ = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), 0
    if rank != 0:
        return 0
    from cnb.utils.cosmology import zeldovich_arrays
    cfg = make_config(args, 1)
    n = cfg.N_BODIES
    pos, vel = zeldovich_arrays(cfg.N_GRID, 1)
    mass = np.full(n, 1.0 / n, np.float32)
    threads = os.cpu_count() or 1
    a = cfg.A_START
    for _ in range(args.warmup):
        cpu_reference_step(pos, vel, mass, a, 0.002, cfg, args.cpu_sample, threads)
    total = 0.0
    wall0 = time.perf_counter()
    for k in range(args.steps):
        pos, vel, s = cpu_reference_step(pos, vel, mass, a, 0.002, cfg, args.cpu_sample, threads)
        a += 0.002
        total += s
    wall = time.perf_counter() - wall0
    value = n * args.steps / total
    check = None
    if 0 < args.cpu_sample < n:
        # the sampled force traversal against the traversal timed on every body, once
        _, _, _, check = cpu_reference_step(pos, vel, mass, a, 0.002, cfg, args.cpu_sample, threads,
                                            full_check=True)
    line = {
        "impl": "reference", "metric": metric_for(args.n_grid), "value": value, "unit": "particle-steps/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Zel'dovich ICs)",
        "config": config_dict(cfg, args),
        "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": threads, "kind": "port",
                         "sample": _sample_text(args.cpu_sample, n)},
        "sampling": {"timed_seconds_actual": wall,
                     "note": ("every stage on every body, nothing extrapolated" if check is None else
                              "ms_per_step is the full step the sample stands for: the force traversal "
                              "of the sampled targets scaled to all bodies (checked below against the "
                              "traversal timed on every body of one step)"),
                     "check": check},
        "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


REF_STAGED = os.path.join(ROOT, "oracle", "_ref")


def _spread21(v):
    """21-bit Morton spread of int64 torch tensors (two zero bits between bits)."""
    v = (v | (v << 32)) & 0x1F00000000FFFF
    v = (v | (v << 16)) & 0x1F0000FF0000FF
    v = (v | (v << 8)) & 0x100F00F00F00F00F
    v = (v | (v << 4)) & 0x10C30C30C30C30C3
    v = (v | (v << 2)) & 0x1249249249249249
    return v


def run_reference_gpu(args):
    """The reference's own Numba kernels on this GPU: src/kernels/*.py of
    Cosmo-NBody, unmodified (staged into oracle/_ref by
    oracle/stage_ref_gpu.sh), launched as its engine launches them
    (src/core/engine.py:55-123, src/core/octree.py:45-83,
    src/core/camera.py:29-48) with torch tensors as the device arrays in place
    of CuPy: stable argsort and gathers by torch (cp.argsort and fancy
    indexing in src/core/state.py:20-40), reset / build_tree /
    compute_multipoles / normalize_com / find_root, the top-tree cache, the
    force traversal in 5 000-body launches (engine.py:91-111), integrate, and
    render_density on the reference's square 1024^2 grid.  One substitution:
    the keys are the 63-bit Morton keys (torch bit interleave of the 21-bit
    coordinates) in place of compute_codes' 30-bit keys of the low 10 bits of
    each coordinate, with which the traversal visits O(N) nodes per body.
    Numba 0.65 compiles for compute capability <= 9.0; its sm_90 PTX is
    JIT-compiled by the driver for the B200."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    base = {"impl": "reference-gpu", "metric": metric_for(args.n_grid)}
    if not os.path.isdir(os.path.join(REF_STAGED, "src", "kernels")):
        print(json.dumps(dict(base, unavailable="reference kernels not staged (oracle/stage_ref_gpu.sh)")))
        return 0
    import types
    import torch
    from numba import cuda
    from cnb.utils.cosmology import zeldovich_arrays
    from cnb.utils.visualizer import get_mvp_matrix
    sys.modules.setdefault("cupy", types.ModuleType("cupy"))   # imported, not used, by render_kernels
    sys.path.insert(0, REF_STAGED)
    from src.kernels.physics_kernels import compute_forces, integrate
    from src.kernels.render_kernels import render_density
    from src.kernels.tree_kernels import (build_top_tree_cache, build_tree, compute_multipoles,
                                          find_root, normalize_com, reset_tree_buffers)
    torch.cuda.set_device(0)
    cfg = make_config(args, 1)
    n = cfg.N_BODIES
    m = 2 * n - 1
    tpb, batch, cache, res = 256, 5000, 256, 1024
    bpg, bpg_nodes = (n + tpb - 1) // tpb, (m + tpb - 1) // tpb
    pos_h, vel_h = zeldovich_arrays(cfg.N_GRID, 1)
    dev = torch.device("cuda", 0)
    pos = [torch.from_numpy(p).to(dev) for p in pos_h]
    vel = [torch.from_numpy(v).to(dev) for v in vel_h]
    mass = torch.full((n,), 1.0 / n, dtype=torch.float32, device=dev)
    child = torch.full((m, 2), -1, dtype=torch.int32, device=dev)
    parent = torch.full((m,), -1, dtype=torch.int32, device=dev)
    root = torch.zeros(1, dtype=torch.int32, device=dev)
    n_mass = torch.zeros(m, dtype=torch.float32, device=dev)
    n_com = torch.zeros((m, 3), dtype=torch.float32, device=dev)
    n_min = torch.zeros((m, 3), dtype=torch.float32, device=dev)
    n_max = torch.zeros((m, 3), dtype=torch.float32, device=dev)
    counters = torch.zeros(m, dtype=torch.int32, device=dev)
    force = torch.zeros((n, 3), dtype=torch.float32, device=dev)
    top_nodes = torch.full((cache,), -1, dtype=torch.int32, device=dev)
    node_to_cache = torch.full((m,), -1, dtype=torch.int32, device=dev)
    grid = torch.zeros((res, res), dtype=torch.float32, device=dev)
    A = cuda.as_cuda_array
    st = {"a": cfg.A_START}

    def step(i):
        a = st["a"]
        H = cfg.H0 * (cfg.OMEGA_M * a ** -3 + cfg.OMEGA_L) ** 0.5
        dt = 0.002 / (a * H) * 0.8
        ix = [torch.clamp((p.double() * 2097152.0).to(torch.int64), 0, 2097151) for p in pos]
        keys = _spread21(ix[0]) | (_spread21(ix[1]) << 1) | (_spread21(ix[2]) << 2)
        order = torch.argsort(keys, stable=True)
        for lst in (pos, vel):
            for k in range(3):
                lst[k] = lst[k][order]
        codes = keys[order].view(torch.uint64)
        reset_tree_buffers[bpg_nodes, tpb](A(child), A(parent), A(counters), A(root))
        build_tree[bpg, tpb](A(codes), A(child), A(parent))
        compute_multipoles[bpg, tpb](A(pos[0]), A(pos[1]), A(pos[2]), A(mass), A(child), A(parent),
                                     A(n_mass), A(n_com), A(n_min), A(n_max), A(counters))
        normalize_com[(m + 255) // 256, 256](A(n_mass), A(n_com), m)
        find_root[bpg_nodes, tpb](A(parent), A(root))
        force.zero_()
        node_to_cache.fill_(-1)
        build_top_tree_cache[1, 1](A(child), A(root), A(top_nodes), A(node_to_cache), cache)
        for off in range(0, n, batch):
            c = min(batch, n - off)
            compute_forces[(c + tpb - 1) // tpb, tpb](
                A(pos[0]), A(pos[1]), A(pos[2]), A(child), A(n_mass), A(n_com), A(n_min), A(n_max),
                A(force), cfg.THETA, cfg.G, cfg.SOFTENING, cfg.BOX_SIZE, A(root), A(top_nodes),
                A(node_to_cache), off)
        integrate[bpg, tpb](A(pos[0]), A(pos[1]), A(pos[2]), A(vel[0]), A(vel[1]), A(vel[2]),
                            A(force), a, H, dt)
        grid.zero_()
        mvp = torch.from_numpy(get_mvp_matrix(i, (0.5, 0.5, 0.5), 1.0, cfg)).to(dev)
        render_density[bpg, tpb](A(pos[0]), A(pos[1]), A(pos[2]), A(grid), A(mvp), res)
        st["a"] = a + 0.002

    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for i in range(args.steps):
        step(args.warmup + i)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    print(json.dumps(dict(base, value=n / (ms * 1e-3), unit="particle-steps/s", n_gpus=1,
                          steps=args.steps, warmup=args.warmup, ms_per_step=ms, higher_is_better=True,
                          dtype="f32 storage, f64 force arithmetic (compiled Numba)",
                          data="synthetic (seeded Zel'dovich ICs)",
                          config=dict(config_dict(cfg, args), splat="1024x1024 (reference square grid)",
                                      keys="63-bit Morton (torch) in place of compute_codes' 30-bit keys",
                                      sort="torch.argsort(stable=True) in place of cp.argsort",
                                      force_launches_per_step=(n + batch - 1) // batch))), flush=True)
    return 0


def config_dict(cfg, args):
    return {"workload": f"Zel'dovich {cfg.N_GRID}^3 plain Barnes-Hut step + {cfg.RES_W}x{cfg.RES_H} splat",
            "n_bodies": cfg.N_BODIES, "theta": cfg.THETA, "softening": cfg.SOFTENING,
            "da": 0.002, "a_start": cfg.A_START, "seed": 1, "keys": "morton63",
            "sort": getattr(cfg, "SORT_MODE", "auto"),
            "force_mode": cfg.FORCE_MODE, "mac": cfg.MAC, "quadrupole": cfg.QUADRUPOLE, "upward": cfg.UPWARD,
            "precision": cfg.PRECISION,
            "bodies_per_lane": cfg.BODIES_PER_LANE, "slab_bodies": cfg.SLAB_BODIES,
            "l2": "flushed between timed steps (256 MB write)", "parallelism": f"replicas x{args.gpus}"}


# ---------------------------------------------------------------- GPU

def run_ours(args):
    import torch
    from cnb import _lib
    from cnb.core.engine import SimulationEngine
    from cnb.core.state import SimulationState
    from cnb.utils.cosmology import zeldovich_arrays

    ws, rank, local = dist_init()
    torch.cuda.set_device(local)
    seed = replica_seed(rank)
    cfg = make_config(args, seed)
    n = cfg.N_BODIES
    pos_h, vel_h = zeldovich_arrays(cfg.N_GRID, seed)
    state = SimulationState(n, pos_h, vel_h)
    eng = SimulationEngine(cfg, state)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def one_step(i):
        eng.step()
        eng.camera.splat(i, *state.pos)

    for i in range(args.warmup):
        one_step(i)
    eng.check()
    tune_report = None
    if args.force_mode == "grouped" and not args.no_tune:
        from cnb import autotune
        tune_report = autotune.tune(eng)          # launch shape for this GPU / workload
    # per-stage breakdown and interaction counts from two eager steps (untimed)
    eng.enable_stage_timing(True)
    eng.stats.zero_()
    for i in range(2):
        one_step(args.warmup + i)
    stages = {k: v / 2 for k, v in eng.stage_times().items()}
    eng.enable_stage_timing(False)
    stats = eng.stats.cpu().numpy()
    interactions_per_step = float(stats[0]) / 2       # body-node interactions
    forces_ms = stages.get("forces", 0.0)
    eng.check()
    step0 = args.warmup + 2
    launches_per_step = None
    if args.graph:
        l0 = _lib.launch_count()
        eng.capture(splat=True)                        # 2 eager steps + a 2-step graph
        launches_per_step = (_lib.launch_count() - l0) // 4   # captured launches are counted once
    sampler = ClockSampler(local) if not args.profile else None
    if sampler:
        sampler.__enter__()
        t_end = time.time() + 1.0                      # pre-roll so the clock samples see load
        while time.time() < t_end:
            eng.replay() if args.graph else one_step(step0)
            torch.cuda.synchronize()
    near0 = state._ctx.stats()[0]
    barrier(ws)
    launches0 = _lib.launch_count()
    # graph mode: one replay = two steps; an odd K ends with one eager device step
    n_iter = (args.steps + 1) // 2 if args.graph else args.steps
    steps_done = args.steps
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(n_iter)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(n_iter)]
    for k in range(n_iter):
        flush.zero_()
        starts[k].record()
        if not args.graph:
            one_step(step0 + k)
        elif 2 * k + 1 < args.steps:
            eng.replay()
        else:
            eng.mvp_slots[0].copy_(eng.camera.mvp_host(eng._graph_step))
            eng._step_device(eng.mvp_slots[0])
            eng.a += eng.da
        ends[k].record()
    barrier(ws)
    if sampler:
        sampler.__exit__()
    if not args.graph:
        launches_per_step = (_lib.launch_count() - launches0) // args.steps
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    total_ms = max_over_ranks(sum(step_ms), ws)
    eng.check()
    value = aggregate_rate(n, steps_done, ws, total_ms)
    args.steps_done = steps_done
    launches = launches_per_step * steps_done
    if args.graph:
        # a captured sort holds the full radix sort (zeroing, histogram, 8 passes) in a
        # conditional node that does not run when the near-sorted path took the sort
        launches -= FULL_SORT_KERNELS * (state._ctx.stats()[0] - near0)

    line = {"metric": metric_for(args.n_grid), "value": value, "unit": "particle-steps/s", "n_gpus": ws,
            "steps": steps_done, "warmup": args.warmup, "ms_per_step": total_ms / steps_done,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded Zel'dovich ICs)", "config": config_dict(cfg, args),
            "gpu_launches": int(launches),
            "gpu_launches_per_step": round(launches / steps_done, 1), "cuda_graph": bool(args.graph),
            "stages_ms_eager": stages}
    if tune_report is not None:
        line["autotune"] = tune_report
    # which sort ran: the near-sorted path or the full radix sort (counts over the whole run)
    from cnb.core.state import sort_mode_for
    near_sorts, full_sorts = state._ctx.stats()
    line["sort"] = {"mode": sort_mode_for(cfg, "morton63"), "near_sorted_path": near_sorts,
                    "full_radix_sort": full_sorts}
    # the launch shape the timed steps used (the autotuner's choice, if it ran)
    line["config"].update(bodies_per_lane=eng.bodies_per_lane, block_warps=eng.block_warps,
                          super_bodies=eng.super_bodies)
    # HBM-bound stages against the measured copy bandwidth, algorithmic bytes per body:
    # keys 20 + sort 20 + permute 60; build 20 + upward/normalise 190; integrate 60
    hbm = measured_peaks()["hbm_gbs"]
    algo = {"sort": 100, "tree": 210, "integrate": 60}
    line["stage_roofline"] = {
        k: {"ms": stages[k], "bytes_per_body": b, "GB/s": n * b / (stages[k] * 1e-3) / 1e9,
            "frac_of_measured_hbm": n * b / (stages[k] * 1e-3) / 1e9 / hbm}
        for k, b in algo.items() if stages.get(k)}
    line["max_node_stack"] = int(eng.tree_manager.workspace[2].item()) if eng.tree_manager.node_table is not None else None
    if args.force_mode == "grouped":
        line["interactions_per_body"] = interactions_per_step / n

    if not args.profile:
        probes = {}
        peak = fma_peak_tflops(probes)
        achieved = interactions_per_step * FLOPS_PER_INTERACTION / (forces_ms * 1e-3) / 1e12
        traffic = FORCES_TRAFFIC_BYTES_128.get(args.mac) if (
            args.n_grid == 128 and abs(args.theta - 0.5) < 1e-9 and args.force_mode == "grouped") else None
        line["roofline"] = {"kernel": FORCES_KERNEL.get(args.mac, "k_forces_ref")
                            if args.force_mode == "grouped" else "k_forces_ref",
                            "bound": "fp32", "achieved": achieved,
                            "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                            "traffic": traffic,
                            "traffic_unit": "bytes per launch",
                            "traffic_source": "ncu capture of this kernel on this workload (one launch, "
                                              "64-body buckets, 512-body super-buckets), not this run"
                                              if traffic else None,
                            "peak_probes_tflops": probes,
                            "note": "peak = measured FP32 FMA throughput, the higher of scalar FFMA "
                                    "(cnb_fma_probe) and packed FFMA2 (cnb_fma2_probe) chains; "
                                    f"{FLOPS_PER_INTERACTION} flops per body-node interaction; "
                                    "interactions = the accepted (body, node) pairs counted on the device"}
        line["clocks"] = sampler.summary()
        line["accuracy"] = accuracy(eng, args)
        line["e2e"] = e2e(eng, args, ws)
        if args.mac == "ref_x" and args.force_mode == "grouped":
            # the reference's test decided once per bucket: finer node sets than the
            # reference's (not its forces), reported beside the headline
            line["variants"] = [variant(eng, args, "ref_x_bucket", flush)]
        if args.learned and args.n_grid == 128 and args.force_mode == "grouped":
            line["learned_vs_plain"] = learned_vs_plain(args, flush)
        if rank == 0:
            line["cpu_baseline"] = cpu_baseline(args)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def variant(eng, args, mac_name, flush):
    """The timed loop of the headline (CUDA-graph replays of two steps with
    splats, L2 flushed between replays) with another opening test, plus its
    interaction count and force error; the engine keeps its launch shape."""
    import torch
    from cnb.core.engine import MACS
    saved = eng.mac
    eng.mac = MACS[mac_name]
    try:
        eng.stats.zero_()
        eng.enable_stage_timing(True)
        for _ in range(2):
            eng.step()
        stages = {k: v / 2 for k, v in eng.stage_times().items()}
        eng.enable_stage_timing(False)
        inter = float(eng.stats[0].item()) / 2 / eng.state.n
        eng.capture(splat=True)
        reps = 5
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(reps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(reps)]
        for k in range(reps):
            flush.zero_()
            starts[k].record()
            eng.replay()
            ends[k].record()
        torch.cuda.synchronize()
        ms = sum(a.elapsed_time(b) for a, b in zip(starts, ends)) / (2 * reps)
        eng.check()
        acc = accuracy(eng, args)
    finally:
        eng.mac = saved
        eng._graph = None
    return {"mac": mac_name, "value": eng.state.n / (ms * 1e-3), "unit": "particle-steps/s",
            "ms_per_step": ms, "steps": 2 * reps, "forces_ms_eager": stages.get("forces"),
            "interactions_per_body": inter, "accuracy": acc}


LEARNED_WEIGHTS = os.path.join(ROOT, "cosmo-nbody_b200", "cnb", "data", "theta_ewald.npz")


def _timed_replays(eng, flush, reps=5):
    """ms per step of `reps` replays of the engine's two-step graph, L2 flushed between."""
    import torch
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(reps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(reps)]
    for k in range(reps):
        flush.zero_()
        starts[k].record()
        eng.replay()
        ends[k].record()
    torch.cuda.synchronize()
    return sum(a.elapsed_time(b) for a, b in zip(starts, ends)) / (2 * reps)


def learned_vs_plain(args, flush):
    """The headline metric's second half: on the evolved 128^3 state (seed 4,
    100 steps of the plain recipe), plain theta = 0.5 against the learned
    per-bucket theta under the periodic (Ewald) law, at matched p99 relative
    force error against the float64 Ewald direct sum on a seeded sample.
    The learned angles (committed weights) are scaled by one factor, bisected
    so that their p99 does not exceed plain's; each arm is then timed as full
    steps (CUDA-graph replays of two steps, L2 flushed).  Also reported: the
    p99 of both arms on every body against a reference-accuracy tree
    (quadrupoles, theta = 0.2), and the bound of any per-bucket policy on this
    state (Lagrangian allocation at plain's p99 on every body)."""
    import torch
    from cnb.controller import ThetaController
    from cnb.core.engine import SimulationEngine
    from cnb.core.state import SimulationState
    from cnb.studies import _cfg, _direct, _errors, _evolve, _reference_tree_forces, lagrangian_bound
    if not os.path.exists(LEARNED_WEIGHTS):
        return {"unavailable": "no trained weights (python -m cnb.studies controller --save ...)"}
    n_grid, steps = 128, 100
    n = n_grid ** 3
    pos, vel, a = _evolve(n_grid, 4, steps)
    cfg = _cfg(n_grid, MAC="ewald", BODIES_PER_LANE=2, BLOCK_WARPS=4, A_START=a,
               A_END=a + 1000 * 0.002, RES=args.width, RES_W=args.width, RES_H=args.height)
    eng = SimulationEngine(cfg, SimulationState(n, pos, vel))
    eng.forces_only()
    plain_acc = eng.state.force.clone()
    ref_tree, qeng, ref_theta = _reference_tree_forces(n_grid, pos, vel, 2)
    targets = np.sort(np.random.default_rng(0).choice(n, args.learned_sample, replace=False)).astype(np.int64)
    t0 = time.time()
    ref = _direct(eng.state, targets, cfg.SOFTENING, periodic=True)
    torch.cuda.synchronize()
    direct_s = time.time() - t0
    ref_self = _errors(qeng.state.force, ref, targets)
    del qeng
    ctl = ThetaController().load(LEARNED_WEIGHTS)

    def evaluate(scale):
        eng.controller = ctl if scale is not None else None
        eng.controller_scale = scale or 1.0
        eng.controller_accel = plain_acc
        if scale is None:
            eng.theta_per_group = None
        eng.stats.zero_()
        eng.compute_forces()
        torch.cuda.synchronize()
        e_all = (eng.state.force.double() - ref_tree).norm(dim=1) / ref_tree.norm(dim=1)
        return dict(_errors(eng.state.force, ref, targets),
                    p99_rel_every_body_vs_tree=float(torch.quantile(e_all.float(), 0.99).item()),
                    interactions_per_body=float(eng.stats[0].item()) / n)

    plain = evaluate(None)
    lo, hi = 0.2, 3.0
    for _ in range(14):
        mid = 0.5 * (lo + hi)
        lo, hi = (mid, hi) if evaluate(mid)["p99_rel"] <= plain["p99_rel"] else (lo, mid)
    learned = evaluate(lo)
    eng.controller_accel = None
    bound = lagrangian_bound(eng, ref_tree)
    bound.pop("theta_allocation")
    out = {}
    for name, scale, errs in (("plain", None, plain), ("learned", lo, learned)):
        eng.controller = ctl if scale is not None else None
        eng.controller_scale = scale or 1.0
        eng.theta_per_group = None
        eng.stats.zero_()
        eng.enable_stage_timing(True)
        for _ in range(2):
            eng.step()
        stages = {k: v / 2 for k, v in eng.stage_times().items()}
        eng.enable_stage_timing(False)
        eng.capture(splat=True)
        ms = _timed_replays(eng, flush)
        eng._graph = None
        out[name] = dict(value=n / (ms * 1e-3), unit="particle-steps/s", ms_per_step=ms,
                         forces_ms_eager=stages.get("forces"), theta="0.5" if scale is None else
                         f"learned, scaled x{scale:.4f}", **errs)
    eng.controller = None
    eng.check()
    return {"workload": f"Zel'dovich {n_grid}^3 seed 4 after {steps} steps (a = {a:.3f}), "
                        "periodic (Ewald) law, monopoles, full step + splat",
            "error": f"|a - a_ref| / |a_ref| against the float64 Ewald direct sum on {targets.size} "
                     f"seeded bodies ({direct_s:.1f} s); the every-body reference is the periodic-law "
                     f"tree with quadrupoles at theta {ref_theta}, p99 {ref_self['p99_rel']:.3g} on "
                     f"that sample",
            "plain": out["plain"], "learned": out["learned"],
            "speedup": out["learned"]["value"] / out["plain"]["value"],
            "interaction_ratio": plain["interactions_per_body"] / learned["interactions_per_body"],
            "bound": bound, "weights": os.path.relpath(LEARNED_WEIGHTS, ROOT)}


def accuracy(eng, args):
    """Median / p99 relative force error against the float64 minimum-image
    direct sum on a seeded random sample of bodies, for the current state."""
    import torch
    from cnb import _lib
    s = eng.state
    eng.forces_only()
    n = s.n
    ewald = eng.mac == _lib.MAC_EWALD
    # the periodic oracle evaluates hundreds of float64 terms per pair: a smaller sample
    k = min(args.accuracy_sample if not ewald else min(args.accuracy_sample, 512), n)
    targets = np.sort(np.random.default_rng(0).choice(n, k, replace=False)).astype(np.int64)
    T = torch.from_numpy(targets).cuda()
    out = torch.empty((k, 3), dtype=torch.float64, device="cuda")
    st = int(torch.cuda.current_stream().cuda_stream)
    _lib.call("cnb_direct_sum_ewald_f64" if ewald else "cnb_direct_sum_f64",
              *(p.data_ptr() for p in s.pos), s.mass.data_ptr(), n, T.data_ptr(),
              k, float(eng.config.G), float(eng.config.SOFTENING), out.data_ptr(), st)
    ref = out.cpu().numpy()
    got = s.force[T].double().cpu().numpy()
    e = np.linalg.norm(got - ref, axis=1) / np.linalg.norm(ref, axis=1)
    rms = np.sqrt((np.linalg.norm(ref, axis=1) ** 2).mean())
    en = np.linalg.norm(got - ref, axis=1) / rms
    vs = "float64 periodic (Ewald) direct sum" if ewald else "float64 minimum-image direct sum"
    return {"vs": vs, "sample": k, "median_rel": float(np.median(e)),
            "p99_rel": float(np.percentile(e, 99)), "p99_rms_normalised": float(np.percentile(en, 99))}


def e2e(eng, args, ws):
    """The same step through the public API with host buffers: every step
    copies positions and velocities in from pinned host memory and copies
    positions, velocities and the density grid back.  `value`: the host-fed
    stepping API (cnb.core.hoststep.HostStepper), whose copies run on their own
    streams under the compute; `serial`: copy in, step, copy out one after
    another on one stream."""
    import torch
    from cnb.core.hoststep import HostStepper
    s = eng.state
    n = s.n
    host_in = [torch.empty(n, dtype=torch.float32, pin_memory=True) for _ in range(6)]
    for h, d in zip(host_in, s.pos + s.vel):
        h.copy_(d)
    host_out = [torch.empty(n, dtype=torch.float32, pin_memory=True) for _ in range(6)]
    grid_h = torch.empty(tuple(eng.camera.grid_d.shape), dtype=torch.float32, pin_memory=True)
    # the first copy-in and the last copy-out of a run overlap nothing: time enough steps
    # that they do not dominate (at 10 steps they add ~0.2 ms per step)
    steps = max(args.steps, E2E_MIN_STEPS)
    main = torch.cuda.current_stream()
    hs = HostStepper(eng)
    for _ in range(2):
        hs.submit(host_in, host_out, grid_h)
    hs.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    hs.h2d.wait_stream(main)          # the first copy-in starts inside the timed region
    for k in range(steps):
        hs.submit(host_in, host_out, grid_h)
    main.wait_stream(hs.d2h)          # ... and the last copy-out ends inside it
    e1.record()
    e1.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1), ws)
    # the same transfers one after another
    torch.cuda.synchronize()
    e0.record()
    for k in range(steps):
        for h, d in zip(host_in, s.pos + s.vel):
            d.copy_(h, non_blocking=True)
        eng.step()
        eng.camera.splat(k, *s.pos)
        for h, d in zip(host_out, s.pos + s.vel):
            h.copy_(d, non_blocking=True)
        grid_h.copy_(eng.camera.grid_d, non_blocking=True)
    e1.record()
    e1.synchronize()
    ms_serial = max_over_ranks(e0.elapsed_time(e1), ws)
    return {"value": ws * n * steps / (ms * 1e-3), "unit": "particle-steps/s", "steps": steps,
            "h2d_bytes_per_step": 24 * n, "d2h_bytes_per_step": 24 * n + 4 * grid_h.numel(),
            "api": "cnb.core.hoststep.HostStepper.submit (SimulationEngine.step + Camera.splat, "
                   "copies on their own streams, two staging slots)",
            "serial": {"value": ws * n * steps / (ms_serial * 1e-3),
                       "api": "copy in, SimulationEngine.step + Camera.splat, copy out on one stream"}}


def cpu_baseline(args):
    from cnb.utils.cosmology import zeldovich_arrays
    cfg = make_config(args, 1)
    n = cfg.N_BODIES
    pos, vel = zeldovich_arrays(cfg.N_GRID, 1)
    mass = np.full(n, 1.0 / n, np.float32)
    threads = os.cpu_count() or 1
    _, _, s = cpu_reference_step(pos, vel, mass, cfg.A_START, 0.002, cfg, args.cpu_sample, threads)
    return {"value": n / s, "unit": "particle-steps/s", "cores": threads, "kind": "port",
            "sample": _sample_text(args.cpu_sample, n)}


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.impl == "reference-gpu":
        return run_reference_gpu(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
