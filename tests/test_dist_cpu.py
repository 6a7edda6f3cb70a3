"""The multi-rank host logic of bench.py on CPU: two gloo ranks, each an
independent box (replicas), job time = max over ranks, aggregate rate over
all ranks' bodies.  The per-rank work is the CPU oracle's step on a tiny
box, so nothing here needs a GPU."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, ws, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        import sys
        root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
        sys.path[:0] = [root, os.path.join(root, "cosmo-nbody_b200")]
        import bench
        from cnb.utils.cosmology import zeldovich_arrays
        from oracle import oracle as orc
        seed = bench.replica_seed(rank)
        pos, vel = zeldovich_arrays(8, seed)
        n = 512
        r = orc.run_reference_step(pos, vel, np.full(n, 1.0 / n, np.float32), 0.02, 0.002, 0.5, 1.0,
                                   0.5 / 8, key_mode=orc.KEY_MORTON63, nthreads=1)
        ms = 10.0 * (rank + 1)                 # stand-in per-rank times: rank 1 is the slowest
        mx = bench.max_over_ranks(ms, ws, device="cpu")
        rate = bench.aggregate_rate(n, 4, ws, mx)
        checksum = float(np.abs(r["force"]).sum())
        t = __import__("torch").tensor([checksum], dtype=__import__("torch").float64)
        gathered = [t.clone() for _ in range(ws)]
        dist.all_gather(gathered, t)
        out[rank] = (seed, mx, rate, [float(g.item()) for g in gathered])
    finally:
        dist.destroy_process_group()


def test_two_replica_ranks_gloo():
    ws = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        ctx = mp.get_context("spawn")
        procs = [ctx.Process(target=_worker, args=(r, ws, port, out)) for r in range(ws)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=180)
            assert p.exitcode == 0
        res = dict(out)
    assert res[0][0] != res[1][0]                     # independent boxes
    assert res[0][1] == res[1][1] == 20.0             # max over ranks
    assert res[0][2] == pytest.approx(2 * 512 * 4 / 0.020)
    assert res[0][3] == res[1][3] and res[0][3][0] != res[0][3][1]   # different replicas' forces
