"""The C-ABI library loads and exports every symbol include/cnb.h declares
(no compute calls: runs without a GPU)."""
import ctypes
import os
import re

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "cnb.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(cnb_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "cnb_compute_codes" in names and "cnb_forces_grouped" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol():
    from cnb import _lib
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    from cnb import _lib
    assert set(declared_functions()) == set(_lib.SIGNATURES), \
        set(declared_functions()) ^ set(_lib.SIGNATURES)


def test_host_only_entry_points():
    from cnb import _lib
    lib = _lib.load()
    assert lib.cnb_version() >= 1
    assert lib.cnb_error_string(_lib.CNB_E_INVALID_ARG) == b"invalid argument"
    # argument validation happens before any device work
    assert lib.cnb_compute_codes(None, None, None, None, None, 10, 0, None) == _lib.CNB_E_INVALID_ARG
    assert lib.cnb_compute_codes(None, None, None, None, None, 0, 0, None) == _lib.CNB_OK
    assert lib.cnb_compute_codes(None, None, None, None, None, -1, 0, None) == _lib.CNB_E_INVALID_ARG
    assert lib.cnb_build_tree(None, None, None, 5, None) == _lib.CNB_E_INVALID_ARG
    assert lib.cnb_forces_grouped(None, None, None, None, None, None, 5, 0.5, None, 7, 1, 4, 1.0,
                                  0.01, 1.0, 0.0, None, None, None) == _lib.CNB_E_INVALID_ARG
    assert lib.cnb_forces_grouped(None, None, None, None, None, None, 5, 0.5, None, 0, 3, 4, 1.0,
                                  0.01, 1.0, 0.0, None, None, None) == _lib.CNB_E_INVALID_ARG
    assert lib.cnb_forces_grouped(None, None, None, None, None, None, 5, 0.5, None, 0, 1, 3, 1.0,
                                  0.01, 1.0, 0.0, None, None, None) == _lib.CNB_E_INVALID_ARG
    assert lib.cnb_make_buckets(None, None, 5, 32, None, None) == _lib.CNB_E_INVALID_ARG
    assert lib.cnb_two_level_workspace_bytes(1000, 16) == -1
    assert lib.cnb_two_level_workspace_bytes(1 << 21, 1024) > 16 * (1 << 21)
    assert lib.cnb_forces_two_level(None, None, None, None, None, None, None, None, 0, 1024, None,
                                    5, 0.5, 0, 1, 8, 1.0, 0.01, 1.0, None, None, None) == _lib.CNB_E_INVALID_ARG
    assert lib.cnb_forces_two_level(None, None, None, None, None, None, None, None, 0, 1024, None,
                                    5, 0.5, 1, 1, 8, 1.0, 0.01, 1.0, None, None, None) == _lib.CNB_E_INVALID_ARG
    assert lib.cnb_sort_pairs(None, None, None, None, None, 5, 30, None) == _lib.CNB_E_INVALID_ARG
    assert lib.cnb_ctx_take_flags(None, None, None) == _lib.CNB_E_INVALID_ARG
    assert lib.cnb_ctx_set_sort_mode(None, _lib.SORT_ADAPTIVE) == _lib.CNB_E_INVALID_ARG
    assert lib.cnb_ctx_inject_sort_faults(None, 10, 3, 0) == _lib.CNB_E_INVALID_ARG
    # sort buffers: the same array in and out is allowed, any other overlap is
    # rejected before the device is touched (these addresses are never read)
    a = 1 << 20
    assert lib.cnb_sort_pairs_noalloc(a, a + 8, None, a + 4096, 10, 63, None) == _lib.CNB_E_INVALID_ARG
    assert lib.cnb_sort_pairs_noalloc(a, a + 4096, a + 8192, a + 8196, 10, 63, None) == _lib.CNB_E_INVALID_ARG
    assert lib.cnb_sort_pairs_noalloc(a, a + 4096, None, a + 40, 10, 63, None) == _lib.CNB_E_INVALID_ARG
    assert lib.cnb_ctx_sort_stats(None, None) == _lib.CNB_E_INVALID_ARG
    assert lib.cnb_render_density(None, None, None, None, None, 4, 0, 4, None) == _lib.CNB_E_INVALID_ARG


def test_launch_objects_validate_shape():
    from cnb.kernels.morton import compute_codes
    with pytest.raises(TypeError):
        compute_codes(1, 2, 3)
    with pytest.raises(TypeError):
        compute_codes[1]
    with pytest.raises(ValueError):
        compute_codes[1, 2048]


def test_launch_objects_reject_host_arrays():
    import numpy as np
    from cnb.kernels.morton import compute_codes
    x = np.zeros(4, np.float32)
    with pytest.raises(TypeError):
        compute_codes[1, 256, 1](x, x, x, np.zeros(4, np.uint64), None, 4)


def test_entry_points_of_the_fused_tree_and_training_validate_arguments():
    """The fused build, the tensor-core gradient and the test hook reject bad
    arguments before any device work."""
    from cnb import _lib
    lib = _lib.load()
    E = _lib.CNB_E_INVALID_ARG
    # fused build: no workspace, no root slot, bad sizes, misaligned tables
    assert lib.cnb_build_tree_buckets(None, None, None, None, None, None, 5, 64, None, 0, None, None) == E
    fake = 1 << 20   # never dereferenced: validation fails first
    assert lib.cnb_build_tree_buckets(None, None, None, None, None, fake, 5, 64, fake, 0, None, None) == E
    assert lib.cnb_build_tree_buckets(fake, fake, fake, fake, fake, fake, 5, 0, fake, 0, None, None) == E
    assert lib.cnb_build_tree_buckets(fake, fake, fake, fake, fake, fake, 5, 64, fake, 0, fake, None) == E
    assert lib.cnb_build_tree_buckets(fake, fake, fake, fake + 4, fake, fake, 5, 64, fake, 512, fake,
                                      None) == E
    assert lib.cnb_build_tree_buckets(fake, fake, fake, fake, fake, fake, -1, 64, fake, 0, None, None) == E
    # tensor-core gradient: scratch size and alignment
    assert lib.cnb_mlp_grad_mma_scratch_bytes(0) == -1
    assert lib.cnb_mlp_grad_mma_scratch_bytes(1) == 416 * 32
    assert lib.cnb_mlp_grad_mma_scratch_bytes(33) == 416 * 64
    nb = lib.cnb_mlp_grad_mma_scratch_bytes(100)
    assert lib.cnb_mlp_grad_mma(fake, fake, 100, fake, 1.0, fake, nb - 16, fake, fake, None) == E
    assert lib.cnb_mlp_grad_mma(fake, fake, 100, fake, 1.0, fake + 8, nb, fake, fake, None) == E
    assert lib.cnb_mlp_grad_mma(fake, fake, 0, fake, 1.0, fake, nb, fake, fake, None) == E
    # the exact traversal's test hook
    assert lib.cnb_exact_test_spill(-1) == E
    assert lib.cnb_exact_test_spill(0) == _lib.CNB_OK
    # two-level forces: ranges and parents both given or both NULL (prebuilt table)
    assert lib.cnb_forces_two_level(fake, fake, fake, fake, fake, None, fake, fake, 1 << 30, 512, fake,
                                    5, 0.5, 0, 2, 2, 1.0, 0.01, 1.0, None, None, None) == E
