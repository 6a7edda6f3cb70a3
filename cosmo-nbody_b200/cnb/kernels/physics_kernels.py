"""Physics kernels (src/kernels/physics_kernels.py of the reference), on libcnb.

`compute_forces` follows the reference's float64 arithmetic;
`compute_forces_f32` is the same traversal in float32.  Both honour `off`
and the thread count of the launch (targets off .. off + grid*block - 1,
clipped to N), so the reference's batched launch loop
(src/core/engine.py:91-111) works unchanged.
"""
import numpy as np

from .. import _lib
from .._arrays import dptr, shape_of, status_buffer
from ._launch import Kernel


def _forces(precision, launch, pos_x, pos_y, pos_z, children, n_mass, n_com, n_min, n_max, force,
            theta, G, soft, box, root, top_nodes, node_to_cache, off):
    n = shape_of(pos_x)[0]
    m = 2 * n - 1
    dptr(top_nodes, np.int32, (-1,), "top_nodes")          # validated, not needed
    dptr(node_to_cache, np.int32, (m,), "node_to_cache")   # validated, not needed
    _lib.call("cnb_compute_forces", dptr(pos_x, np.float32, (n,), "pos_x"),
              dptr(pos_y, np.float32, (n,), "pos_y"), dptr(pos_z, np.float32, (n,), "pos_z"),
              dptr(children, np.int32, (m, 2), "children"), dptr(n_mass, np.float32, (m,), "n_mass"),
              dptr(n_com, np.float32, (m, 3), "n_com"), dptr(n_min, np.float32, (m, 3), "n_min"),
              dptr(n_max, np.float32, (m, 3), "n_max"), dptr(force, np.float32, (n, 3), "force"),
              float(theta), float(G), float(soft), float(box), dptr(root, np.int32, (-1,), "root"),
              int(off), launch.threads, n, precision, status_buffer().data_ptr(), launch.stream)


def _forces64(launch, *args):
    """physics_kernels.py:14-153 compute_forces(pos_x, pos_y, pos_z, children, n_mass, n_com,
    n_min, n_max, force, theta, G, soft, box, root, top_nodes, node_to_cache, off)."""
    _forces(_lib.PREC_F64, launch, *args)


def _forces32(launch, *args):
    """compute_forces in float32 arithmetic."""
    _forces(_lib.PREC_F32, launch, *args)


def _integrate(launch, pos_x, pos_y, pos_z, vel_x, vel_y, vel_z, force, a, H, dt):
    """physics_kernels.py:155-203 integrate(pos_x, pos_y, pos_z, vel_x, vel_y, vel_z, force, a,
    H, dt)."""
    n = shape_of(pos_x)[0]
    if launch.threads < n:
        raise ValueError(f"integrate: launch of {launch.threads} threads does not cover {n} bodies")
    _lib.call("cnb_integrate", *(dptr(v, np.float32, (n,), nm) for v, nm in
                                 ((pos_x, "pos_x"), (pos_y, "pos_y"), (pos_z, "pos_z"),
                                  (vel_x, "vel_x"), (vel_y, "vel_y"), (vel_z, "vel_z"))),
              dptr(force, np.float32, (n, 3), "force"), n, float(a), float(H), float(dt),
              launch.stream)


compute_forces = Kernel("compute_forces", _forces64)
compute_forces_f32 = Kernel("compute_forces_f32", _forces32)
integrate = Kernel("integrate", _integrate)
