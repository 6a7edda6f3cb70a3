"""Topology validation: valid Karras trees pass, corrupted ones (made on the
host) and the invalid trees long runs of equal 30-bit keys produce under the
reference's tie rule are flagged."""
import numpy as np
import pytest

from oracle import oracle as orc

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _validate(children, parents):
    from cnb import _lib
    n = (children.shape[0] + 1) // 2
    C = torch.from_numpy(np.ascontiguousarray(children, np.int32)).cuda()
    P = torch.from_numpy(np.ascontiguousarray(parents, np.int32)).cuda()
    scratch = torch.empty(2 * n, dtype=torch.int32, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    _lib.call("cnb_validate_tree", C.data_ptr(), P.data_ptr(), n, scratch.data_ptr(), status.data_ptr(),
              int(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    return int(status.item())


def test_valid_trees_pass():
    from cnb.utils.cosmology import zeldovich_arrays
    for ng, mode in ((16, 0), (32, 1), (2, 1)):
        (x, y, z), _ = zeldovich_arrays(ng, 0)
        codes, _ = orc.compute_codes(x, y, z, mode)
        ch, par = orc.build_tree(codes[orc.argsort_stable(codes)])
        assert _validate(ch, par) == 0


def test_corrupted_trees_are_flagged():
    from cnb.utils.cosmology import zeldovich_arrays
    (x, y, z), _ = zeldovich_arrays(8, 1)
    codes, _ = orc.compute_codes(x, y, z, 1)
    ch, par = orc.build_tree(codes[orc.argsort_stable(codes)])
    n = codes.size
    bad = ch.copy()
    bad[n + 5, 0] = bad[n + 9, 1]          # a node claimed twice
    assert _validate(bad, par) != 0
    badp = par.copy()
    badp[3] = -1                           # two roots
    assert _validate(ch, badp) != 0
    bad2 = ch.copy()
    bad2[n + 1, 1] = 10 ** 7               # child index out of range
    assert _validate(bad2, par) != 0


def test_long_equal_key_runs_flagged():
    rng = np.random.default_rng(11)
    keys = np.sort(rng.integers(0, 64, 3000, dtype=np.uint64))
    ch, par = orc.build_tree(keys)
    assert _validate(ch, par) != 0
