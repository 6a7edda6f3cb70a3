"""cnb -- B200 (sm_100a) Barnes-Hut step behind the reference's Python
interfaces.

Module map (reference -> here):
  src/kernels/morton.py          -> cnb.kernels.morton
  src/kernels/tree_kernels.py    -> cnb.kernels.tree_kernels
  src/kernels/physics_kernels.py -> cnb.kernels.physics_kernels
  src/kernels/render_kernels.py  -> cnb.kernels.render_kernels
  src/core/state.py              -> cnb.core.state
  src/core/octree.py             -> cnb.core.octree
  src/core/engine.py             -> cnb.core.engine
  src/core/camera.py             -> cnb.core.camera
  src/utils/config.py            -> cnb.utils.config
  src/utils/cosmology.py         -> cnb.utils.cosmology
  src/utils/visualizer.py        -> cnb.utils.visualizer
Every kernel runs in libcnb.so (C ABI in include/cnb.h); there is no CPU
fallback.
"""
from ._lib import CnbError, load  # noqa: F401

__version__ = "0.1.0"
