"""The adaptive sort (CNB_SORT_ADAPTIVE): the near-sorted path and the full
radix sort it falls back to return the stable argsort of the keys
(src/core/state.py:35 `cp.argsort(codes)`), bit-exact against numpy's stable
argsort, on every kind of input order: already sorted, a few keys displaced
near or far, displaced runs, ties, tile edges, random and reversed (the
fallback), inside a CUDA graph whose input changes between replays, and on
the keys of a simulated step."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

TILE = 4096


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from cnb import _lib
    _lib.load()


def lib():
    from cnb import _lib
    return _lib


def stream():
    return int(torch.cuda.current_stream().cuda_stream)


class Ctx:
    def __init__(self, n, mode=1):
        self.p = C.c_void_p()
        lib().call("cnb_ctx_create", n, C.byref(self.p))
        lib().call("cnb_ctx_set_sort_mode", self.p, mode)

    def stats(self):
        out = (C.c_int64 * 2)()
        lib().call("cnb_ctx_sort_stats", self.p, out)
        return int(out[0]), int(out[1])

    def flags(self):
        f = torch.zeros(1, dtype=torch.int32, device="cuda")
        lib().call("cnb_ctx_take_flags", self.p, f.data_ptr(), stream())
        return int(f.item())

    def __del__(self):
        lib().load().cnb_ctx_destroy(self.p)


def sort(ctx, keys, bits=63):
    n = keys.size
    K = torch.from_numpy(keys.view(np.int64).copy()).cuda().view(torch.uint64)
    Ko = torch.zeros_like(K)
    P = torch.zeros(n, dtype=torch.uint32, device="cuda")
    lib().call("cnb_sort_pairs", ctx.p, K.data_ptr(), Ko.data_ptr(), None, P.data_ptr(), n, bits,
               stream())
    torch.cuda.synchronize()
    return Ko.cpu().numpy().view(np.uint64), P.cpu().numpy()


def check(ctx, keys, bits=63):
    before = ctx.stats()
    sk, perm = sort(ctx, keys, bits)
    want = np.argsort(keys, kind="stable")
    np.testing.assert_array_equal(perm.astype(np.int64), want)
    np.testing.assert_array_equal(sk, keys[want])
    assert ctx.flags() == 0
    after = ctx.stats()
    return "near" if after[0] > before[0] else "full"


def sorted_keys(n, seed, bits=63):
    rng = np.random.default_rng(seed)
    return np.sort(rng.integers(0, 1 << bits, n, dtype=np.uint64))


def jump(keys, src, dst):
    """Moves the key at src to dst (the rest shift): a body that crossed the
    periodic boundary, or overtook many neighbours."""
    k = keys[src]
    rest = np.delete(keys, src)
    return np.insert(rest, dst, k)


def test_sorted_and_tiny_inputs_take_the_near_path():
    ctx = Ctx(1 << 21)
    for n in (1, 2, 3, 100, TILE - 1, TILE, TILE + 1, 3 * TILE + 17, 1 << 21):
        assert check(ctx, sorted_keys(n, n)) == "near", n


def test_displaced_keys_near_and_far():
    ctx = Ctx(1 << 21)
    n = 1 << 21
    rng = np.random.default_rng(1)
    base = sorted_keys(n, 2)
    # adjacent swaps
    k = base.copy()
    sw = rng.integers(0, n - 1, 300)
    k[sw], k[sw + 1] = k[sw + 1].copy(), k[sw].copy()
    assert check(ctx, k) == "near"
    # keys moved far forward and far backward, some onto tile edges
    k = base.copy()
    for src, dst in ((5, n - 3), (n - 2, 0), (TILE - 1, 7 * TILE), (9 * TILE, TILE),
                     (12345, 12345 + 200), (777777, 700000)):
        k = jump(k, src, dst)
    assert check(ctx, k) == "near"
    # keys replaced by values far away (wrapped coordinates)
    k = base.copy()
    idx = rng.integers(0, n, 200)
    k[idx] = rng.integers(0, 1 << 63, 200, dtype=np.uint64)
    assert check(ctx, k) == "near"


@pytest.mark.parametrize("run", [2, 5, 40, 127, 300])
def test_displaced_runs(run):
    """Neighbours that move together (a clump crossing the boundary): runs of
    ascending keys dropped far from their place, across tile edges too."""
    ctx = Ctx(1 << 20)
    n = 1 << 20
    k = sorted_keys(n, run)
    blk = k[1000:1000 + run].copy()
    k = np.insert(np.delete(k, np.s_[1000:1000 + run]), n - run - TILE // 2 - run // 2, blk)
    blk = k[5 * TILE - run // 2:5 * TILE - run // 2 + run].copy()
    k = np.insert(np.delete(k, np.s_[5 * TILE - run // 2:5 * TILE - run // 2 + run]), 10, blk)
    path = check(ctx, k)
    if run <= 127:
        assert path == "near"


def test_ties_keep_input_order():
    ctx = Ctx(1 << 18)
    n = 1 << 18
    rng = np.random.default_rng(3)
    k = np.sort(rng.integers(0, 1000, n, dtype=np.uint64))  # long runs of equal keys
    sw = rng.integers(0, n - 1, 100)
    k[sw], k[sw + 1] = k[sw + 1].copy(), k[sw].copy()
    k = jump(k, 10, n - 10)
    assert check(ctx, k) == "near"
    # all keys equal, and equal keys displaced among equal keys
    assert check(ctx, np.full(n, 42, np.uint64)) == "near"
    k = np.full(n, 42, np.uint64)
    k[rng.integers(0, n, 50)] = 7
    assert check(ctx, k) == "near"


@pytest.mark.parametrize("kind", ["random", "reversed", "many_swaps", "swaps_in_every_tile"])
def test_unsorted_inputs_fall_back_to_the_full_sort(kind):
    ctx = Ctx(1 << 21)
    n = 1 << 21
    rng = np.random.default_rng(4)
    if kind == "random":
        k = rng.integers(0, 1 << 63, n, dtype=np.uint64)
    elif kind == "reversed":
        k = sorted_keys(n, 5)[::-1].copy()
    elif kind == "many_swaps":
        k = sorted_keys(n, 6)
        sw = rng.integers(0, n - 1, 5000)  # more displaced keys than the path takes
        k[sw], k[sw + 1] = k[sw + 1].copy(), k[sw].copy()
    else:
        k = sorted_keys(n, 7)
        sw = np.arange(0, n - 1, 200)  # twenty displaced keys in every tile
        k[sw], k[sw + 1] = k[sw + 1].copy(), k[sw].copy()
    assert check(ctx, k) == "full"


def test_cap_boundary_is_exact_either_way():
    ctx = Ctx(1 << 21)
    n = 1 << 21
    rng = np.random.default_rng(8)
    for swaps in (1500, 2040, 2048, 2049, 2100, 3000):
        k = sorted_keys(n, swaps)
        sw = np.sort(rng.choice(np.arange(0, n - 1, 3), swaps, replace=False))
        k[sw], k[sw + 1] = k[sw + 1].copy(), k[sw].copy()
        check(ctx, k)


def test_full_mode_never_takes_the_near_path():
    ctx = Ctx(1 << 16, mode=0)
    assert check(ctx, sorted_keys(1 << 16, 9)) == "full"


def test_graph_replay_follows_the_input():
    """The path is chosen on the device: one captured graph sorts a
    near-sorted input on the near path and a random input on the full sort."""
    n = 1_000_003
    ctx = Ctx(n)
    near = jump(sorted_keys(n, 10), 3, n - 5)
    rand = np.random.default_rng(11).integers(0, 1 << 63, n, dtype=np.uint64)
    K = torch.from_numpy(near.view(np.int64).copy()).cuda().view(torch.uint64)
    Ko = torch.zeros_like(K)
    P = torch.zeros(n, dtype=torch.uint32, device="cuda")
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        st = int(s.cuda_stream)
        lib().call("cnb_sort_pairs", ctx.p, K.data_ptr(), Ko.data_ptr(), None, P.data_ptr(), n, 63, st)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            lib().call("cnb_sort_pairs", ctx.p, K.data_ptr(), Ko.data_ptr(), None, P.data_ptr(), n,
                       63, int(s.cuda_stream))
    torch.cuda.current_stream().wait_stream(s)
    for keys, path in ((near, "near"), (rand, "full"), (near, "near")):
        K.copy_(torch.from_numpy(keys.view(np.int64).copy()).cuda().view(torch.uint64))
        P.zero_()
        before = ctx.stats()
        g.replay()
        torch.cuda.synchronize()
        want = np.argsort(keys, kind="stable")
        np.testing.assert_array_equal(P.cpu().numpy().astype(np.int64), want)
        after = ctx.stats()
        assert (after[0] > before[0]) == (path == "near")
    assert ctx.flags() == 0


def test_step_keys_take_the_near_path():
    """Keys of 64^3 Zel'dovich bodies sorted at one step, recomputed after
    the drift of the next (the order the step sees)."""
    from cnb.utils.cosmology import zeldovich_arrays
    from oracle import oracle as orc
    (pos, vel) = zeldovich_arrays(64, 1)
    p = [np.asarray(a, np.float64) for a in pos]
    v = [np.asarray(a, np.float64) for a in vel]
    c0, _ = orc.compute_codes(*[a.astype(np.float32) for a in p], orc.KEY_MORTON63)
    order = np.argsort(c0, kind="stable")
    a = 0.02
    dt = 0.98 / 2500 / (a * orc.hubble(a)) * 0.8
    ctx = Ctx(64 ** 3)
    for steps in (1, 5, 20):
        q = [((p[i] + steps * v[i] * dt / a) % 1.0).astype(np.float32)[order] for i in range(3)]
        c1, _ = orc.compute_codes(*q, orc.KEY_MORTON63)
        assert check(ctx, c1) == "near"


def test_engine_adaptive_matches_full():
    """Eight morton63 steps with the adaptive sort and with the full sort:
    identical state."""
    from cnb.core.engine import SimulationEngine
    from cnb.core.state import SimulationState
    from cnb.utils import config as cfgmod
    from cnb.utils.cosmology import zeldovich_arrays
    out = {}
    for mode in ("adaptive", "full"):
        cfg = cfgmod.make(N_GRID=32, KEY_MODE="morton63", SORT_MODE=mode, FORCE_MODE="grouped",
                          BODIES_PER_LANE=2, BLOCK_WARPS=2, THETA=0.5)
        pos, vel = zeldovich_arrays(32, 5)
        state = SimulationState(32 ** 3, pos, vel)
        eng = SimulationEngine(cfg, state, camera=False)
        for _ in range(8):
            eng.step()
        eng.check()
        torch.cuda.synchronize()
        out[mode] = [t.cpu().numpy().copy() for t in state.pos + state.vel]
        st = state._ctx.stats()
        if mode == "adaptive":
            assert st[0] >= 6, st  # the first sort (lattice order) falls back
        else:
            assert st[0] == 0
    for a, b in zip(out["adaptive"], out["full"]):
        np.testing.assert_array_equal(a, b)
