"""cnb_sort_pairs_noalloc: the radix sort for callers that cannot allocate
device memory (e.g. a plugin whose host application owns all device memory
through its own pool).  It must give exactly the same sorted keys and
permutation as cnb_sort_pairs, which sorts with context-owned scratch, on
two calls in a row (the fixed scratch array keeps the previous call's
contents, which must not leak into the next result), and must refuse sizes
beyond its stated maximum.  Collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _sort_both(keys, bits, vals=None):
    from cnb import _lib
    n = keys.size
    st = int(torch.cuda.current_stream().cuda_stream)
    K = torch.from_numpy(keys).cuda()
    V = torch.from_numpy(vals).cuda() if vals is not None else None
    vptr = V.data_ptr() if V is not None else None
    ko_a = torch.empty_like(K)
    po_a = torch.empty(n, dtype=torch.uint32, device="cuda")
    ctx = C.c_void_p()
    _lib.call("cnb_ctx_create", n, C.byref(ctx))
    try:
        _lib.call("cnb_sort_pairs", ctx, K.data_ptr(), ko_a.data_ptr(), vptr, po_a.data_ptr(), n, bits, st)
        torch.cuda.synchronize()
    finally:
        _lib.load().cnb_ctx_destroy(ctx)
    ko_b = torch.empty_like(K)
    po_b = torch.empty(n, dtype=torch.uint32, device="cuda")
    _lib.call("cnb_sort_pairs_noalloc", K.data_ptr(), ko_b.data_ptr(), vptr, po_b.data_ptr(), n, bits, st)
    torch.cuda.synchronize()
    return (ko_a.cpu().numpy(), po_a.cpu().numpy()), (ko_b.cpu().numpy(), po_b.cpu().numpy())


def test_noalloc_sort_matches_context_sort_twice():
    from cnb import _lib
    rng = np.random.default_rng(2024)
    # first call: near the maximum, 63-bit keys with duplicates
    n1 = (1 << 20) - 5
    k1 = rng.integers(0, 1 << 63, n1, dtype=np.uint64)
    k1[rng.integers(0, n1, n1 // 7)] = k1[3]
    a, b = _sort_both(k1, 63)
    np.testing.assert_array_equal(b[0], a[0])
    np.testing.assert_array_equal(b[1], a[1])
    # second call, smaller and with carried values: stale scratch must not matter
    n2 = 70001
    k2 = rng.integers(0, 1 << 30, n2, dtype=np.uint64)
    v2 = rng.permutation(n2).astype(np.uint32)
    a, b = _sort_both(k2, 30, v2)
    np.testing.assert_array_equal(b[0], a[0])
    np.testing.assert_array_equal(b[1], a[1])
    assert np.all(np.diff(b[0].astype(np.int64)) >= 0)


def _noalloc(K, ko, V, po, n, bits):
    from cnb import _lib
    st = int(torch.cuda.current_stream().cuda_stream)
    _lib.call("cnb_sort_pairs_noalloc", K.data_ptr(), ko.data_ptr(), V.data_ptr() if V is not None else None,
              po.data_ptr(), n, bits, st)
    torch.cuda.synchronize()


def test_noalloc_sort_edge_shapes():
    """The largest size (the last tile fills the scratch), one 8-bit pass with
    distinct buffers, one pass in place (keys_out == keys_in, then two passes
    run), and perm_out == idx_in: every result equals numpy's stable argsort."""
    rng = np.random.default_rng(77)
    n = 1 << 20
    keys = rng.integers(0, 1 << 63, n, dtype=np.uint64)
    a, b = _sort_both(keys, 63)
    np.testing.assert_array_equal(b[1].astype(np.int64), np.argsort(keys, kind="stable"))
    np.testing.assert_array_equal(b[0], a[0])
    for n, in_place in ((100_003, False), (4096 * 3 + 17, True)):
        k = rng.integers(0, 256, n, dtype=np.uint64)
        want = np.argsort(k, kind="stable")
        K = torch.from_numpy(k).cuda()
        ko = K if in_place else torch.empty_like(K)
        po = torch.empty(n, dtype=torch.uint32, device="cuda")
        _noalloc(K, ko, None, po, n, 8)
        np.testing.assert_array_equal(po.cpu().numpy().astype(np.int64), want)
        np.testing.assert_array_equal(ko.cpu().numpy(), k[want])
    # carried indices sorted in place of themselves
    n = 50_001
    k = rng.integers(0, 256, n, dtype=np.uint64)
    v = rng.permutation(n).astype(np.uint32)
    K = torch.from_numpy(k).cuda()
    V = torch.from_numpy(v).cuda()
    ko = torch.empty_like(K)
    _noalloc(K, ko, V, V, n, 8)
    want = np.argsort(k, kind="stable")
    np.testing.assert_array_equal(V.cpu().numpy(), v[want])
    np.testing.assert_array_equal(ko.cpu().numpy(), k[want])


def test_noalloc_sort_rejects_oversize():
    from cnb import _lib
    lib = _lib.load()
    big = (1 << 20) + 1
    rc = lib.cnb_sort_pairs_noalloc(None, None, None, None, big, 63, None)
    assert rc == _lib.CNB_E_TOO_LARGE
    assert lib.cnb_error_string(rc) == b"size exceeds the supported maximum"
