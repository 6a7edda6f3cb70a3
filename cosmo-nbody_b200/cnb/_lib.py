"""ctypes binding of libcnb.so (declarations in include/cnb.h).

The library is built in-tree by ``cosmo-nbody_b200/build.py``.  There is no
fallback: if the library cannot be loaded, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcnb.so")

CNB_OK = 0
CNB_E_INVALID_ARG = -1
CNB_E_CUDA = -2
CNB_E_NO_MEMORY = -3
CNB_E_TOO_LARGE = -4
CNB_E_DEVICE_FLAG = -5

FLAG_STACK_OVERFLOW = 1
FLAG_BAD_TOPOLOGY = 2
FLAG_NONFINITE = 4
FLAG_LIST_OVERFLOW = 8
FLAG_WAIT_LIMIT = 16
FLAG_SORT_CHECK = 32

KEY_COMPAT30 = 0
KEY_MORTON63 = 1
MAC_REF_X = 0
MAC_PERIODIC = 1
MAC_EWALD = 2
MAC_REF_X_BUCKET = 3
SORT_FULL = 0
SORT_ADAPTIVE = 1
SORT_NEAR_CAP = 2048
PREC_F32 = 0
PREC_F64 = 1
UPWARD_PLAIN = 0
UPWARD_COMPENSATED = 1
MLP_PARAMS = 5057

_p = C.c_void_p
_i64 = C.c_int64
_i32 = C.c_int32
_int = C.c_int
_d = C.c_double
_f = C.c_float

# name -> (restype, argtypes); must match include/cnb.h
SIGNATURES = {
    "cnb_version": (_int, []),
    "cnb_error_string": (C.c_char_p, [_int]),
    "cnb_last_cuda_error": (_int, []),
    "cnb_launch_count": (_i64, []),
    "cnb_compute_codes": (_int, [_p, _p, _p, _p, _p, _i64, _int, _p]),
    "cnb_ctx_create": (_int, [_i64, C.POINTER(_p)]),
    "cnb_ctx_destroy": (_int, [_p]),
    "cnb_sort_pairs": (_int, [_p, _p, _p, _p, _p, _i64, _int, _p]),
    "cnb_sort_pairs_noalloc": (_int, [_p, _p, _p, _p, _i64, _int, _p]),
    "cnb_ctx_set_sort_mode": (_int, [_p, _int]),
    "cnb_ctx_inject_sort_faults": (_int, [_p, _i32, _i64, _i64]),
    "cnb_ctx_sort_stats": (_int, [_p, _p]),
    "cnb_ctx_take_flags": (_int, [_p, _p, _p]),
    "cnb_gather_f32": (_int, [_p, _int, _p, _p, _i64, _p]),
    "cnb_reset_tree_buffers": (_int, [_p, _p, _p, _p, _i64, _p]),
    "cnb_build_tree": (_int, [_p, _p, _p, _i64, _p]),
    "cnb_compute_multipoles": (_int, [_p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _i64, _p, _p]),
    "cnb_upward": (_int, [_p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _i64, _int, _p, _p, _p]),
    "cnb_normalize_com": (_int, [_p, _p, _i64, _p]),
    "cnb_validate_tree": (_int, [_p, _p, _i64, _p, _p, _p]),
    "cnb_upward_table": (_int, [_p, _p, _p, _p, _p, _p, _p, _p, _p, _i64, _p, _p]),
    "cnb_unpack_nodes": (_int, [_p, _p, _p, _p, _p, _i64, _p]),
    "cnb_find_root": (_int, [_p, _p, _i64, _p]),
    "cnb_build_top_tree_cache": (_int, [_p, _p, _p, _p, _i32, _p]),
    "cnb_compute_forces": (_int, [_p, _p, _p, _p, _p, _p, _p, _p, _p, _d, _d, _d, _d, _p, _i64,
                                  _i64, _i64, _int, _p, _p]),
    "cnb_integrate": (_int, [_p, _p, _p, _p, _p, _p, _p, _i64, _d, _d, _d, _p]),
    "cnb_render_density": (_int, [_p, _p, _p, _p, _p, _i64, _int, _int, _p]),
    "cnb_pack_nodes": (_int, [_p, _p, _p, _p, _p, _p, _i64, _p]),
    "cnb_build_tree_ranges": (_int, [_p, _p, _p, _p, _i64, _p]),
    "cnb_make_buckets": (_int, [_p, _p, _i64, _int, _p, _p]),
    "cnb_build_tree_buckets": (_int, [_p, _p, _p, _p, _p, _p, _i64, _int, _p, _int, _p, _p]),
    "cnb_forces_grouped": (_int, [_p, _p, _p, _p, _p, _p, _i64, _d, _p, _int, _int, _int, _d, _d, _d,
                                  _d, _p, _p, _p]),
    "cnb_two_level_workspace_bytes": (_i64, [_i64, _int]),
    "cnb_forces_two_level": (_int, [_p, _p, _p, _p, _p, _p, _p, _p, _i64, _int, _p, _i64, _d, _int,
                                    _int, _int, _d, _d, _d, _p, _p, _p]),
    "cnb_make_buckets_boxes": (_int, [_p, _p, _p, _int, _i64, _int, _p, _p]),
    "cnb_compute_codes_boxes": (_int, [_p, _p, _p, _p, _p, _i64, _int, _p]),
    "cnb_box_roots": (_int, [_p, _p, _p, _int, _i64, _int, _p, _p]),
    "cnb_forces_grouped_boxes": (_int, [_p, _p, _p, _p, _p, _p, _i64, _p, _int, _p, _p, _p, _int, _int,
                                        _int, _d, _p, _p, _p]),
    "cnb_integrate_boxes": (_int, [_p, _p, _p, _p, _p, _p, _p, _p, _int, _i64, _p, _p]),
    "cnb_bucket_features": (_int, [_p, _p, _p, _i64, _p, _p, _p, _int, _p]),
    "cnb_controller_theta": (_int, [_p, _p, _p, _i64, _p, _p, _p, _p, _int, _p]),
    "cnb_mlp_predict": (_int, [_p, _int, _p, _p, _p]),
    "cnb_mlp_grad": (_int, [_p, _p, _int, _p, _f, _p, _p, _p, _p]),
    "cnb_mlp_grad_mma_scratch_bytes": (_i64, [_int]),
    "cnb_mlp_grad_mma": (_int, [_p, _p, _int, _p, _f, _p, _i64, _p, _p, _p]),
    "cnb_adam_step": (_int, [_p, _p, _p, _p, _int, _f, _f, _f, _f, _int, _p]),
    "cnb_to_bf16": (_int, [_p, _p, _int, _p]),
    "cnb_colorize": (_int, [_p, _int, _int, _p, _p, _p, _p]),
    "cnb_ewald_table": (_int, [_p, _int, _p]),
    "cnb_forces_grouped_ewald": (_int, [_p, _p, _p, _p, _p, _p, _i64, _d, _p, _int, _int, _d, _d, _p,
                                        _int, _p, _p, _p, _p, _p, _p]),
    "cnb_order_buckets": (_int, [_p, _p, _p, _p]),
    "cnb_upward_table_quad": (_int, [_p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _i64, _p, _p]),
    "cnb_upward_table_buckets": (_int, [_p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _i64, _p, _p]),
    "cnb_direct_sum_ewald_f64": (_int, [_p, _p, _p, _p, _i64, _p, _i64, _d, _d, _p, _p]),
    "cnb_forces_grouped_boxes_ewald": (_int, [_p, _p, _p, _p, _p, _p, _i64, _p, _int, _p, _p, _p, _int,
                                              _int, _d, _p, _int, _p, _p, _p, _p]),
    "cnb_direct_sum_f64": (_int, [_p, _p, _p, _p, _i64, _p, _i64, _d, _d, _p, _p]),
    "cnb_fma_probe": (_int, [_p, _i64, _int, _p]),
    "cnb_fma2_probe": (_int, [_p, _i64, _int, _p]),
    "cnb_exact_test_spill": (_int, [_int]),
}

_lib = None
_lock = threading.Lock()


class CnbError(RuntimeError):
    """Error returned by a libcnb entry point or flagged by a kernel."""

    def __init__(self, msg, code=None, flags=0):
        super().__init__(msg)
        self.code = code
        self.flags = flags


def load():
    """Load libcnb.so once and bind every declared entry point."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise CnbError(f"libcnb.so not built ({LIB_PATH}); run cosmo-nbody_b200/build.py")
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def check(rc, what):
    """Raise CnbError for a non-zero return code of entry point `what`."""
    if rc != CNB_OK:
        lib = load()
        msg = lib.cnb_error_string(rc).decode()
        if rc == CNB_E_CUDA:
            msg += f" (cudaError {lib.cnb_last_cuda_error()})"
        raise CnbError(f"{what}: {msg}", code=rc)
    return rc


def call(name, *args):
    """Call entry point `name` and raise on a non-zero return code."""
    return check(getattr(load(), name)(*args), name)


def launch_count():
    return int(load().cnb_launch_count())
