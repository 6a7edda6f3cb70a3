"""The fused upward pass (sums + traversal table in one kernel) writes the same
bits as the separate upward, normalisation and packing kernels."""
import numpy as np
import pytest

from oracle import oracle as orc

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _tree(n_grid, seed):
    from cnb.utils.cosmology import zeldovich_arrays
    (x, y, z), _ = zeldovich_arrays(n_grid, seed)
    codes, _ = orc.compute_codes(x, y, z, 1)
    perm = orc.argsort_stable(codes)
    return [a[perm] for a in (x, y, z)], codes[perm]


@pytest.mark.parametrize("n_grid", [2, 16, 32])
def test_fused_table_equals_separate_passes(n_grid):
    from cnb import _lib
    pos, codes = _tree(n_grid, 3)
    n = codes.size
    m = 2 * n - 1
    st = int(torch.cuda.current_stream().cuda_stream)
    K = torch.from_numpy(codes).cuda()
    P = [torch.from_numpy(a).cuda() for a in pos]
    M = torch.full((n,), 1.0 / n, device="cuda")
    ch = torch.full((m, 2), -1, dtype=torch.int32, device="cuda")
    par = torch.full((m,), -1, dtype=torch.int32, device="cuda")
    _lib.call("cnb_build_tree", K.data_ptr(), ch.data_ptr(), par.data_ptr(), n, st)

    def bufs():
        return [torch.zeros(m, device="cuda"), torch.zeros((m, 3), device="cuda"),
                torch.zeros((m, 3), device="cuda"), torch.zeros((m, 3), device="cuda"),
                torch.zeros(m, dtype=torch.int32, device="cuda")]

    a = bufs()
    _lib.call("cnb_upward", *(p.data_ptr() for p in P), M.data_ptr(), ch.data_ptr(), par.data_ptr(),
              *(t.data_ptr() for t in a[:4]), None, a[4].data_ptr(), n, 0, None, None, st)
    table_a = torch.empty((4, m, 4), device="cuda")
    _lib.call("cnb_pack_nodes", *(t.data_ptr() for t in a[:4]), ch.data_ptr(), table_a.data_ptr(), m, st)
    b = bufs()
    table_b = torch.empty((4, m, 4), device="cuda")
    sums = torch.empty((m, 4), device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    _lib.call("cnb_upward_table", *(p.data_ptr() for p in P), M.data_ptr(), ch.data_ptr(), par.data_ptr(),
              b[4].data_ptr(), table_b.data_ptr(), sums.data_ptr(), n, status.data_ptr(), st)
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    np.testing.assert_array_equal(table_a.cpu().numpy().view(np.uint32), table_b.cpu().numpy().view(np.uint32))
    # the reference-layout arrays unpacked from the table are the reference's values
    _lib.call("cnb_unpack_nodes", table_b.data_ptr(), *(t.data_ptr() for t in b[:4]), m, st)
    wm, wc, wlo, whi = orc.compute_multipoles(*pos, M.cpu().numpy(), ch.cpu().numpy(), par.cpu().numpy())
    np.testing.assert_array_equal(b[0].cpu().numpy(), wm)
    np.testing.assert_array_equal(b[1].cpu().numpy(), wc)
    np.testing.assert_array_equal(b[2].cpu().numpy(), wlo)
    np.testing.assert_array_equal(b[3].cpu().numpy(), whi)


def test_octree_manager_grouped_buffers_are_reference_layout():
    from cnb.core.octree import OctreeManager
    pos, codes = _tree(16, 4)
    n = codes.size
    P = [torch.from_numpy(a).cuda() for a in pos]
    M = torch.full((n,), 1.0 / n, device="cuda")
    tm = OctreeManager(n, node_table=True)
    tm.build(P, M, torch.from_numpy(codes).cuda())
    buf = tm.get_buffers()
    ch, par = orc.build_tree(codes)
    wm, wc, wlo, whi = orc.compute_multipoles(*pos, M.cpu().numpy(), ch, par)
    np.testing.assert_array_equal(buf["com"].cpu().numpy(), wc)
    np.testing.assert_array_equal(buf["min"].cpu().numpy(), wlo)
    assert int(buf["root"].item()) == n


@pytest.mark.parametrize("n_grid,bucket", [(2, 32), (16, 32), (32, 64), (24, 16)])
def test_bucketed_upward_equals_one_pass(n_grid, bucket):
    """cnb_upward_table_buckets (warp per bucket, shared-memory counters, then
    the levels above) writes the same bits as the one-pass cnb_upward_table,
    with and without second moments."""
    from cnb import _lib
    pos, codes = _tree(n_grid, 7)
    n = codes.size
    m = 2 * n - 1
    st = int(torch.cuda.current_stream().cuda_stream)
    K = torch.from_numpy(codes).cuda()
    P = [torch.from_numpy(a).cuda() for a in pos]
    M = torch.full((n,), 1.0 / n, device="cuda")
    ch = torch.full((m, 2), -1, dtype=torch.int32, device="cuda")
    par = torch.full((m,), -1, dtype=torch.int32, device="cuda")
    rg = torch.zeros((max(n - 1, 1), 2), dtype=torch.int32, device="cuda")
    _lib.call("cnb_build_tree_ranges", K.data_ptr(), ch.data_ptr(), par.data_ptr(), rg.data_ptr(), n, st)
    ws = torch.zeros(4 + 4 * n, dtype=torch.int32, device="cuda")
    _lib.call("cnb_make_buckets", rg.data_ptr(), par.data_ptr(), n, bucket, ws.data_ptr(), st)
    for quad in (False, True):
        out = []
        for entry in ("one", "buckets"):
            table = torch.zeros((4, m, 4), device="cuda")
            sums = torch.zeros((m, 4), device="cuda")
            q = torch.zeros((m, 8), device="cuda") if quad else None
            counts = torch.zeros(m, dtype=torch.int32, device="cuda")
            status = torch.zeros(1, dtype=torch.int32, device="cuda")
            qp = q.data_ptr() if quad else None
            if entry == "one" and quad:
                _lib.call("cnb_upward_table_quad", *(p.data_ptr() for p in P), M.data_ptr(), ch.data_ptr(),
                          par.data_ptr(), counts.data_ptr(), table.data_ptr(), sums.data_ptr(), qp, n,
                          status.data_ptr(), st)
            elif entry == "one":
                _lib.call("cnb_upward_table", *(p.data_ptr() for p in P), M.data_ptr(), ch.data_ptr(),
                          par.data_ptr(), counts.data_ptr(), table.data_ptr(), sums.data_ptr(), n,
                          status.data_ptr(), st)
            else:
                _lib.call("cnb_upward_table_buckets", *(p.data_ptr() for p in P), M.data_ptr(), ch.data_ptr(),
                          par.data_ptr(), ws.data_ptr(), counts.data_ptr(), table.data_ptr(), sums.data_ptr(),
                          qp, n, status.data_ptr(), st)
            torch.cuda.synchronize()
            assert int(status.item()) == 0
            out.append((table.cpu().numpy(), q.cpu().numpy()[n:] if quad else None))
        np.testing.assert_array_equal(out[0][0].view(np.uint32), out[1][0].view(np.uint32))
        if quad:
            np.testing.assert_array_equal(out[0][1].view(np.uint32), out[1][1].view(np.uint32))


def test_bucketed_upward_flags_corrupted_topology():
    """Faults made on the host in a valid tree: a node that is its own parent,
    a leaf whose parent lies outside its bucket, and a bucket above the 64
    bodies the shared-memory pass handles.  Every climb is bounded, so each
    ends with a flag instead of a hang."""
    from cnb import _lib
    pos, codes = _tree(16, 8)
    n = codes.size
    m = 2 * n - 1
    st = int(torch.cuda.current_stream().cuda_stream)
    K = torch.from_numpy(codes).cuda()
    P = [torch.from_numpy(a).cuda() for a in pos]
    M = torch.full((n,), 1.0 / n, device="cuda")
    ch = torch.full((m, 2), -1, dtype=torch.int32, device="cuda")
    par0 = torch.full((m,), -1, dtype=torch.int32, device="cuda")
    rg = torch.zeros((n - 1, 2), dtype=torch.int32, device="cuda")
    _lib.call("cnb_build_tree_ranges", K.data_ptr(), ch.data_ptr(), par0.data_ptr(), rg.data_ptr(), n, st)
    ws = torch.zeros(4 + 4 * n, dtype=torch.int32, device="cuda")
    _lib.call("cnb_make_buckets", rg.data_ptr(), par0.data_ptr(), n, 64, ws.data_ptr(), st)
    torch.cuda.synchronize()
    bk = ws[4:4 + 4 * int(ws[0].item())].view(-1, 4).cpu().numpy()
    big = bk[np.argmax(bk[:, 1])]
    assert big[1] >= 2

    def run(par, work):
        # every buffer stays referenced until the kernels have run
        status = torch.zeros(1, dtype=torch.int32, device="cuda")
        counts = torch.zeros(m, dtype=torch.int32, device="cuda")
        table = torch.zeros((4, m, 4), device="cuda")
        sums = torch.zeros((m, 4), device="cuda")
        _lib.call("cnb_upward_table_buckets", *(p.data_ptr() for p in P), M.data_ptr(), ch.data_ptr(),
                  par.data_ptr(), work.data_ptr(), counts.data_ptr(), table.data_ptr(), sums.data_ptr(),
                  None, n, status.data_ptr(), st)
        torch.cuda.synchronize()
        return int(status.item())

    assert run(par0, ws) == 0
    # an internal node of a bucket that is its own parent
    par = par0.clone()
    inner = int(par0[int(big[0])].item())
    par[inner] = inner
    assert run(par, ws) & _lib.FLAG_BAD_TOPOLOGY
    # a leaf whose parent lies outside its bucket
    par = par0.clone()
    par[int(big[0])] = n  # the tree's root: not in any bucket of several bodies
    assert run(par, ws) & _lib.FLAG_BAD_TOPOLOGY
    # a bucket table with buckets of up to 128 bodies
    ws128 = torch.zeros_like(ws)
    _lib.call("cnb_make_buckets", rg.data_ptr(), par0.data_ptr(), n, 128, ws128.data_ptr(), st)
    torch.cuda.synchronize()
    if int(ws128[4:4 + 4 * int(ws128[0].item())].view(-1, 4)[:, 1].max().item()) > 64:
        assert run(par0, ws128) & _lib.FLAG_LIST_OVERFLOW
