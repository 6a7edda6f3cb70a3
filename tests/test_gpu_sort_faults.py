"""Failure paths of the sort, made to happen without a GPU fault.

The one-sweep radix sort is the only kernel whose blocks wait on one another
(each 4096-key tile looks back at the digit counts that earlier tiles
publish).  Every such wait is bounded; a wait that gives up raises
CNB_FLAG_WAIT_LIMIT and the kernel returns.  The test hook
cnb_ctx_inject_sort_faults makes one tile keep its counts to itself (a flag
that nothing sets) and shortens the limit, so the tiles after it give up
within microseconds; the call must return, the flag must reach the caller's
status word through cnb_ctx_take_flags, and after the hook is reset the same
context must sort correctly again.

The near-sorted path checks every destination before it writes; the hook
shifts the destinations past the end of the array, every write must be
skipped (the output keeps its previous contents) and CNB_FLAG_SORT_CHECK must
be raised."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


class Ctx:
    def __init__(self, n):
        from cnb import _lib
        self.lib = _lib
        self.p = C.c_void_p()
        _lib.call("cnb_ctx_create", n, C.byref(self.p))

    def close(self):
        self.lib.load().cnb_ctx_destroy(self.p)


def _stream():
    return int(torch.cuda.current_stream().cuda_stream)


def _sort(ctx, keys, bits=63):
    from cnb import _lib
    n = keys.size
    K = torch.from_numpy(keys).cuda()
    ko = torch.from_numpy(np.full(n, 7, np.uint64)).cuda()
    po = torch.from_numpy(np.full(n, 0xFFFFFFFF, np.uint32)).cuda()
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    _lib.call("cnb_sort_pairs", ctx.p, K.data_ptr(), ko.data_ptr(), None, po.data_ptr(), n, bits,
              _stream())
    _lib.call("cnb_ctx_take_flags", ctx.p, status.data_ptr(), _stream())
    torch.cuda.synchronize()
    return int(status.item()), ko.cpu().numpy(), po.cpu().numpy()


def test_lookback_wait_gives_up_and_reports():
    from cnb import _lib
    rng = np.random.default_rng(11)
    n = 40 * 4096 + 123
    keys = rng.integers(0, 1 << 63, n, dtype=np.uint64)
    ctx = Ctx(n)
    try:
        _lib.call("cnb_ctx_set_sort_mode", ctx.p, _lib.SORT_FULL)
        _lib.call("cnb_ctx_inject_sort_faults", ctx.p, 256, 3, 0)
        flags, _, _ = _sort(ctx, keys)
        assert flags & _lib.FLAG_WAIT_LIMIT
        # the flag was taken: a second take reports nothing new
        status = torch.zeros(1, dtype=torch.int32, device="cuda")
        _lib.call("cnb_ctx_take_flags", ctx.p, status.data_ptr(), _stream())
        torch.cuda.synchronize()
        assert int(status.item()) == 0
        # hook off: the same context sorts exactly again
        _lib.call("cnb_ctx_inject_sort_faults", ctx.p, 0, -1, 0)
        flags, ko, po = _sort(ctx, keys)
        assert flags == 0
        want = np.argsort(keys, kind="stable")
        np.testing.assert_array_equal(po.astype(np.int64), want)
        np.testing.assert_array_equal(ko, keys[want])
    finally:
        ctx.close()


def test_short_limit_alone_keeps_results_or_reports():
    """A short limit without a withheld tile: the sort either finishes every
    wait in time (exact result, no flag) or reports the give-up -- never a
    wrong result without the flag."""
    from cnb import _lib
    rng = np.random.default_rng(12)
    n = 300 * 4096
    keys = rng.integers(0, 1 << 63, n, dtype=np.uint64)
    ctx = Ctx(n)
    try:
        _lib.call("cnb_ctx_inject_sort_faults", ctx.p, 4, -1, 0)
        flags, ko, po = _sort(ctx, keys)
        if not flags & _lib.FLAG_WAIT_LIMIT:
            np.testing.assert_array_equal(po.astype(np.int64), np.argsort(keys, kind="stable"))
    finally:
        ctx.close()


def test_near_sorted_destination_check():
    from cnb import _lib
    rng = np.random.default_rng(13)
    n = 20 * 4096
    keys = np.sort(rng.integers(0, 1 << 62, n, dtype=np.uint64))
    # a few displaced keys: the near-sorted path applies
    idx = rng.choice(n, 50, replace=False)
    keys[idx] = rng.integers(0, 1 << 62, 50, dtype=np.uint64)
    ctx = Ctx(n)
    try:
        _lib.call("cnb_ctx_set_sort_mode", ctx.p, _lib.SORT_ADAPTIVE)
        _lib.call("cnb_ctx_inject_sort_faults", ctx.p, 0, -1, n)
        flags, ko, po = _sort(ctx, keys)
        assert flags & _lib.FLAG_SORT_CHECK
        # every destination was past the end: nothing was written
        assert (ko == 7).all()
        assert (po == 0xFFFFFFFF).all()
        _lib.call("cnb_ctx_inject_sort_faults", ctx.p, 0, -1, 0)
        flags, ko, po = _sort(ctx, keys)
        assert flags == 0
        np.testing.assert_array_equal(po.astype(np.int64), np.argsort(keys, kind="stable"))
        out = (C.c_int64 * 2)()
        _lib.call("cnb_ctx_sort_stats", ctx.p, out)
        assert out[0] == 2 and out[1] == 0   # both sorts took the near-sorted path
    finally:
        ctx.close()
