"""Tree kernels (src/kernels/tree_kernels.py of the reference), on libcnb.

Same names, argument order and array layouts as the reference:
children [M,2] int32, parents [M] int32, n_mass [M], n_com/n_min/n_max
[M,3] float32, counters [M] int32, root_idx [1] int32, M = 2N - 1.
"""
import numpy as np

from .. import _lib
from .._arrays import dptr, shape_of, status_buffer
from ._launch import Kernel


def _need(launch, work, name):
    if launch.threads < work:
        raise ValueError(f"{name}: launch of {launch.threads} threads does not cover {work} items")


def _reset(launch, child, parent, counters, root_idx):
    """tree_kernels.py:236-262 reset_tree_buffers(child, parent, counters, root_idx)."""
    m = shape_of(child)[0]
    _need(launch, m, "reset_tree_buffers")
    _lib.call("cnb_reset_tree_buffers", dptr(child, np.int32, (m, 2), "child"),
              dptr(parent, np.int32, (m,), "parent"), dptr(counters, np.int32, (m,), "counters"),
              dptr(root_idx, np.int32, (-1,), "root_idx"), m, launch.stream)


def _build(launch, codes, children, parents):
    """tree_kernels.py:60-129 build_tree(codes, children, parents)."""
    n = shape_of(codes)[0]
    m = max(2 * n - 1, 1)
    _need(launch, n - 1, "build_tree")
    _lib.call("cnb_build_tree", dptr(codes, np.uint64, (n,), "codes"),
              dptr(children, np.int32, (m, 2), "children"), dptr(parents, np.int32, (m,), "parents"),
              n, launch.stream)


def _multipoles(launch, pos_x, pos_y, pos_z, mass, children, parents, n_mass, n_com, n_min, n_max,
                counts):
    """tree_kernels.py:131-191 compute_multipoles(...)."""
    n = shape_of(pos_x)[0]
    m = 2 * n - 1
    _need(launch, n, "compute_multipoles")
    _lib.call("cnb_compute_multipoles", dptr(pos_x, np.float32, (n,), "pos_x"),
              dptr(pos_y, np.float32, (n,), "pos_y"), dptr(pos_z, np.float32, (n,), "pos_z"),
              dptr(mass, np.float32, (n,), "mass"), dptr(children, np.int32, (m, 2), "children"),
              dptr(parents, np.int32, (m,), "parents"), dptr(n_mass, np.float32, (m,), "n_mass"),
              dptr(n_com, np.float32, (m, 3), "n_com"), dptr(n_min, np.float32, (m, 3), "n_min"),
              dptr(n_max, np.float32, (m, 3), "n_max"), dptr(counts, np.int32, (m,), "counts"), n,
              status_buffer().data_ptr(), launch.stream)


def _normalize(launch, n_mass, n_com, n_nodes):
    """tree_kernels.py:193-214 normalize_com(n_mass, n_com, n_nodes)."""
    m = min(int(n_nodes), shape_of(n_mass)[0], launch.threads)
    _lib.call("cnb_normalize_com", dptr(n_mass, np.float32, (-1,), "n_mass"),
              dptr(n_com, np.float32, (-1, 3), "n_com"), m, launch.stream)


def _find_root(launch, parents, root_idx):
    """tree_kernels.py:216-234 find_root(parents, root_idx)."""
    m = shape_of(parents)[0]
    _need(launch, m, "find_root")
    _lib.call("cnb_find_root", dptr(parents, np.int32, (m,), "parents"),
              dptr(root_idx, np.int32, (-1,), "root_idx"), m, launch.stream)


def _top_cache(launch, child, root_idx, top_nodes, node_to_cache, cache_size):
    """tree_kernels.py:264-313 build_top_tree_cache(child, root_idx, top_nodes, node_to_cache,
    cache_size)."""
    m = shape_of(child)[0]
    c = int(cache_size)
    if shape_of(top_nodes)[0] < c:
        raise ValueError("top_nodes shorter than cache_size")
    _lib.call("cnb_build_top_tree_cache", dptr(child, np.int32, (m, 2), "child"),
              dptr(root_idx, np.int32, (-1,), "root_idx"), dptr(top_nodes, np.int32, (-1,), "top_nodes"),
              dptr(node_to_cache, np.int32, (m,), "node_to_cache"), c, launch.stream)


reset_tree_buffers = Kernel("reset_tree_buffers", _reset)
build_tree = Kernel("build_tree", _build)
compute_multipoles = Kernel("compute_multipoles", _multipoles)
normalize_com = Kernel("normalize_com", _normalize)
find_root = Kernel("find_root", _find_root)
build_top_tree_cache = Kernel("build_top_tree_cache", _top_cache)
