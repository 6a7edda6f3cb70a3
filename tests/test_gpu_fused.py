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
    """Faults made on the host in a valid tree: an internal node of a bucket
    that is its own child, a node whose child lies outside its bucket, two
    internal nodes that are each other's child (a cycle the counters never
    complete), a bucket root that is its own parent, and a bucket above the
    64 bodies the shared-memory pass handles.  The bucket's topology is
    checked before it is used and every climb is bounded, so each ends with
    a flag instead of a hang."""
    from cnb import _lib
    pos, codes = _tree(16, 8)
    n = codes.size
    m = 2 * n - 1
    st = int(torch.cuda.current_stream().cuda_stream)
    K = torch.from_numpy(codes).cuda()
    P = [torch.from_numpy(a).cuda() for a in pos]
    M = torch.full((n,), 1.0 / n, device="cuda")
    ch0 = torch.full((m, 2), -1, dtype=torch.int32, device="cuda")
    par0 = torch.full((m,), -1, dtype=torch.int32, device="cuda")
    rg = torch.zeros((n - 1, 2), dtype=torch.int32, device="cuda")
    _lib.call("cnb_build_tree_ranges", K.data_ptr(), ch0.data_ptr(), par0.data_ptr(), rg.data_ptr(), n, st)
    ws = torch.zeros(4 + 4 * n, dtype=torch.int32, device="cuda")
    _lib.call("cnb_make_buckets", rg.data_ptr(), par0.data_ptr(), n, 64, ws.data_ptr(), st)
    torch.cuda.synchronize()
    bk = ws[4:4 + 4 * int(ws[0].item())].view(-1, 4).cpu().numpy()
    big = bk[np.argmax(bk[:, 1])]
    assert big[1] >= 8
    root = int(big[2])
    ch_h = ch0.cpu().numpy()

    def run(ch, par, work):
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

    assert run(ch0, par0, ws) == 0
    # an internal node of the bucket that is its own child (in place of one of its children)
    ch = ch0.clone()
    ch[root, 1] = root
    assert run(ch, par0, ws) & _lib.FLAG_BAD_TOPOLOGY
    # a node whose child lies outside its bucket (the tree's root)
    ch = ch0.clone()
    ch[root, 0] = n
    assert run(ch, par0, ws) & _lib.FLAG_BAD_TOPOLOGY
    # two internal nodes of the bucket that are each other's child: every slot
    # keeps one parent, but the cycle is never completed
    a, b = int(ch_h[root, 0]), int(ch_h[root, 1])
    if a >= n and b >= n and ch_h[a, 0] >= 0 and ch_h[b, 0] >= 0:
        ch = ch0.clone()
        ch[a, 0], ch[b, 0] = b, a
        ch[root, 0], ch[root, 1] = int(ch_h[a, 0]), int(ch_h[b, 0])
        assert run(ch, par0, ws) & _lib.FLAG_BAD_TOPOLOGY
    # a bucket root that is its own parent (read by the climb above the buckets)
    par = par0.clone()
    par[root] = root
    assert run(ch0, par, ws) & _lib.FLAG_BAD_TOPOLOGY
    # a bucket table with buckets of up to 128 bodies
    ws128 = torch.zeros_like(ws)
    _lib.call("cnb_make_buckets", rg.data_ptr(), par0.data_ptr(), n, 128, ws128.data_ptr(), st)
    torch.cuda.synchronize()
    if int(ws128[4:4 + 4 * int(ws128[0].item())].view(-1, 4)[:, 1].max().item()) > 64:
        assert run(ch0, par0, ws128) & _lib.FLAG_LIST_OVERFLOW


def _codes_cases():
    rng = np.random.default_rng(11)
    dup = np.sort(rng.integers(0, 1 << 12, 5000).astype(np.uint64))   # many equal keys
    wide = np.sort(rng.integers(0, 1 << 62, 20000, dtype=np.int64).astype(np.uint64))
    return {"one": np.zeros(1, np.uint64), "two": np.array([3, 3], np.uint64),
            "three": np.array([1, 5, 9], np.uint64), "dup": dup, "wide": wide,
            "zeldovich32": _tree(32, 5)[1]}


@pytest.mark.parametrize("case", ["one", "two", "three", "dup", "wide", "zeldovich32"])
@pytest.mark.parametrize("bucket,super_size", [(32, 0), (64, 512), (16, 64)])
def test_fused_build_equals_separate_launches(case, bucket, super_size):
    """cnb_build_tree_buckets writes the children, parents, ranges and root of
    cnb_reset_tree_buffers + cnb_build_tree_ranges + cnb_find_root, zeroes
    the internal nodes' counters, and its bucket and super-bucket tables
    hold the buckets of cnb_make_buckets (same rows, any order)."""
    from cnb import _lib
    codes = _codes_cases()[case]
    n = codes.size
    m = 2 * n - 1
    st = int(torch.cuda.current_stream().cuda_stream)
    K = torch.from_numpy(codes).cuda()

    def tables(fused):
        ch = torch.full((m, 2), -1, dtype=torch.int32, device="cuda")
        par = torch.full((m,), -1, dtype=torch.int32, device="cuda")
        rg = torch.zeros((max(n - 1, 1), 2), dtype=torch.int32, device="cuda")
        cnt = torch.full((m,), 7, dtype=torch.int32, device="cuda")
        root = torch.full((1,), -5, dtype=torch.int32, device="cuda")
        ws = torch.full((4 + 4 * n,), 9, dtype=torch.int32, device="cuda")
        sws = torch.full((4 + 4 * n,), 9, dtype=torch.int32, device="cuda") if super_size else None
        if fused:
            _lib.call("cnb_build_tree_buckets", K.data_ptr(), ch.data_ptr(), par.data_ptr(), rg.data_ptr(),
                      cnt.data_ptr(), root.data_ptr(), n, bucket, ws.data_ptr(), super_size,
                      sws.data_ptr() if sws is not None else None, st)
        else:
            _lib.call("cnb_reset_tree_buffers", ch.data_ptr(), par.data_ptr(), cnt.data_ptr(),
                      root.data_ptr(), m, st)
            _lib.call("cnb_build_tree_ranges", K.data_ptr(), ch.data_ptr(), par.data_ptr(), rg.data_ptr(), n, st)
            _lib.call("cnb_find_root", par.data_ptr(), root.data_ptr(), m, st)
            _lib.call("cnb_make_buckets", rg.data_ptr(), par.data_ptr(), n, bucket, ws.data_ptr(), st)
            if sws is not None:
                _lib.call("cnb_make_buckets", rg.data_ptr(), par.data_ptr(), n, super_size, sws.data_ptr(), st)
        torch.cuda.synchronize()

        def rows(w):
            if w is None:
                return None
            w = w.cpu().numpy()
            r = w[4:4 + 4 * int(w[0])].reshape(-1, 4)
            return w[:4].copy(), r[np.lexsort(r.T[::-1])]
        return (ch.cpu().numpy(), par.cpu().numpy(), rg.cpu().numpy(), int(root.item()),
                cnt.cpu().numpy(), rows(ws), rows(sws))

    a, b = tables(False), tables(True)
    for x, y in zip(a[:3], b[:3]):
        np.testing.assert_array_equal(x, y)
    assert not b[4][n:].any()
    if (a[1] == -1).sum() > 1:
        # equal keys under the reference's tie rule left nodes without a parent
        # (the reference's find_root then returns any of them): the buckets still
        # tile the bodies by range, but some body inside a bucket is no child of
        # the bucket's nodes, and the bucketed upward pass says so
        assert case == "dup"
        P = [torch.rand(n, device="cuda") for _ in range(3)]
        M = torch.full((n,), 1.0 / n, device="cuda")
        ch = torch.from_numpy(b[0]).cuda()
        par = torch.from_numpy(b[1]).cuda()
        ws = torch.from_numpy(np.concatenate([b[5][0], b[5][1].ravel()])).cuda()
        status = torch.zeros(1, dtype=torch.int32, device="cuda")
        cnt = torch.zeros(m, dtype=torch.int32, device="cuda")
        table = torch.zeros((4, m, 4), device="cuda")
        sums = torch.zeros((m, 4), device="cuda")
        _lib.call("cnb_upward_table_buckets", *(p.data_ptr() for p in P), M.data_ptr(), ch.data_ptr(),
                  par.data_ptr(), ws.data_ptr(), cnt.data_ptr(), table.data_ptr(), sums.data_ptr(),
                  None, n, status.data_ptr(), st)
        torch.cuda.synchronize()
        assert int(status.item()) & _lib.FLAG_BAD_TOPOLOGY
        return
    assert a[3] == b[3] == (n if n > 1 else 0)
    check = np.uint32(n * (n + 1) // 2 % (1 << 32)).view(np.int32)
    for ta, tb in zip(a[5:], b[5:]):
        if ta is None:
            continue
        np.testing.assert_array_equal(ta[0], tb[0])
        np.testing.assert_array_equal(ta[1], tb[1])
        assert tb[0][3] == check
    # buckets tile the bodies
    cover = np.zeros(n, np.int32)
    for lo, size, _, _ in b[5][1]:
        cover[lo:lo + size] += 1
    assert (cover == 1).all()


@pytest.mark.parametrize("n_grid,bucket", [(16, 32), (32, 64)])
def test_fused_octree_build_equals_unfused(n_grid, bucket):
    """OctreeManager's fused build (one build launch + the bucketed upward
    pass) gives the node table, tree and root of the launch-by-launch path,
    over repeated builds of moving bodies."""
    from cnb.core.octree import OctreeManager
    pos, codes = _tree(n_grid, 9)
    n = codes.size
    P = [torch.from_numpy(a).cuda() for a in pos]
    M = torch.full((n,), 1.0 / n, device="cuda")
    K = torch.from_numpy(codes).cuda()
    fused = OctreeManager(n, node_table=True, bucket=bucket)
    plain = OctreeManager(n, node_table=True, bucket=bucket)
    assert fused._fused_build
    for step in range(2):
        fused.build(P, M, K)
        plain.bucket = 128  # above 64: the launch-by-launch path (one-pass upward)
        plain.build(P, M, K)
        plain.bucket = bucket
        torch.cuda.synchronize()
        np.testing.assert_array_equal(fused.node_table.cpu().numpy().view(np.uint32),
                                      plain.node_table.cpu().numpy().view(np.uint32))
        np.testing.assert_array_equal(fused.child.cpu().numpy(), plain.child.cpu().numpy())
        np.testing.assert_array_equal(fused.parent.cpu().numpy(), plain.parent.cpu().numpy())
        assert int(fused.root_idx.item()) == int(plain.root_idx.item()) == n
        # the next build: bodies moved, keys re-sorted
        rng = np.random.default_rng(step)
        moved = [(a + rng.normal(0, 1e-3, a.size).astype(np.float32)) % np.float32(1.0) for a in pos]
        c2, _ = orc.compute_codes(*moved, 1)
        perm = orc.argsort_stable(c2)
        P = [torch.from_numpy(a[perm]).cuda() for a in moved]
        K = torch.from_numpy(c2[perm]).cuda()
