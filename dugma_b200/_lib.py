"""ctypes binding of libdugma_b200.so (declarations in include/dugma.h).

The shared library is built in-tree (python -m dugma_b200.build).  Loading
never falls back to anything else: a missing or unloadable library raises.
"""
from __future__ import annotations

import ctypes
import os

from . import build as _build

_LIB = None

c_int, c_double, c_float, c_void_p, c_size_t = ctypes.c_int, ctypes.c_double, ctypes.c_float, ctypes.c_void_p, ctypes.c_size_t
P = ctypes.POINTER
dp = P(c_double)
fp = P(c_float)
ip = P(c_int)
PtrArray = c_void_p * 6

# status codes (dugma.h)
OK, ERR_ARG, ERR_CUDA, ERR_NONPD, ERR_TIMEOUT, ERR_NOMEM, ERR_NUMERIC, ERR_STATE = range(8)
MODEL_REF, MODEL_CONV, MODEL_REF_F64 = 0, 1, 2
DRIVE_REFERENCE, DRIVE_DIRECT = 0, 1

EXPORTS = {
    "dugma_init": (c_int, [dp, dp, dp, dp, dp, c_int, c_int, c_int, PtrArray]),
    "dugma_update_sig": (c_int, [PtrArray, dp, dp, dp, dp, dp, fp]),
    "dugma_compi": (c_int, [PtrArray, dp, dp, dp, dp, dp, dp, dp]),
    "dugma_compi_range": (c_int, [PtrArray, dp, dp, c_double, c_int, c_int, c_int, c_int, dp]),
    "dugma_fr_m": (c_int, [PtrArray]),
    "dugma_last_error": (ctypes.c_char_p, []),
    "dugma_energy": (c_int, [PtrArray, dp, dp, c_double, c_int, dp]),
    "dugma_energy_grad": (c_int, [PtrArray, dp, dp, c_double, c_int, dp, dp, dp]),
    "dugma_energy_grad_range": (c_int, [PtrArray, dp, dp, c_double, c_int, c_int, c_int, dp, dp]),
    "dugma_energy_fd_grad": (c_int, [PtrArray, dp, dp, c_double, c_int, c_double, dp, dp]),
    "dugma_nn": (c_int, [PtrArray, dp, dp, c_int, ip, fp]),
    "dugma_sigma": (c_int, [PtrArray, dp, dp, dp]),
    "dugma_sigma_range": (c_int, [PtrArray, dp, dp, c_int, c_int, dp]),
    "dugma_energy_grad_async": (c_int, [PtrArray, c_void_p, c_int, c_void_p, c_void_p, c_void_p]),
    "dugma_energy_async": (c_int, [PtrArray, c_void_p, c_int, c_void_p, c_void_p]),
    "dugma_autotune": (c_int, [PtrArray, c_int, c_int, ctypes.c_char_p, c_size_t]),
    "dugma_graph_create": (c_int, [PtrArray, c_int, P(c_void_p)]),
    "dugma_graph_eval": (c_int, [c_void_p, dp, dp, c_double, dp, dp]),
    "dugma_graph_destroy": (c_int, [c_void_p]),
    "dugma_em_graph_create": (c_int, [PtrArray, P(c_void_p)]),
    "dugma_em_step": (c_int, [c_void_p, dp, dp, fp, dp]),
    "dugma_em_graph_destroy": (c_int, [c_void_p]),
    "dugma_batch_create": (c_int, [c_int, c_int, ip, ip, P(dp), P(dp), P(dp), P(dp), P(c_void_p)]),
    "dugma_batch_energy_grad": (c_int, [c_void_p, c_int, dp, c_int, dp]),
    "dugma_batch_destroy": (c_int, [c_void_p]),
    "dugma_batch_shapes": (c_int, [ip, c_int]),
    "dugma_batch_set_shape": (c_int, [c_void_p, c_int, c_int, c_int, c_int]),
    "dugma_batch_get_shape": (c_int, [c_void_p, ip]),
    "dugma_batch_autotune": (c_int, [c_void_p, c_int, dp, ctypes.c_char_p, c_size_t]),
    "dugma_batch_timing": (c_int, [c_void_p, c_int, dp, ip]),
    "dugma_register": (c_int, [dp, dp, dp, dp, c_int, c_int, c_int, dp, dp, c_int, c_double, c_double, c_double,
                               c_int, dp, dp, dp]),
    "dugma_version": (ctypes.c_char_p, []),
    "dugma_timing": (c_int, [PtrArray, c_int, dp, ip]),
    "dugma_shapes": (c_int, [c_int, ip, c_int]),
    "dugma_knn_covariance": (c_int, [dp, c_int, c_int, c_int, c_double, c_double, dp]),
    "dugma_minimise_surrogate": (c_int, [c_int, dp, dp, dp, dp, ip]),
    "dugma_energy_grad_noalloc": (c_int, [c_void_p] * 6 + [c_int, c_int, c_int, c_void_p, c_void_p, c_void_p]),
    "dugma_set_shape": (c_int, [PtrArray, c_int, c_int, c_int, c_int, c_int]),
    "dugma_get_shape": (c_int, [PtrArray, c_int, ip]),
    "dugma_calibrate": (c_int, [c_int, dp, dp]),
    "dugma_wait_selftest": (c_int, [c_int, ip]),
    "dugma_coef_work_grid": (c_int, [c_int, c_int, c_int, ip]),
}


class DugmaError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"dugma error {code}: {msg}")
        self.code = code


def lib_path() -> str:
    return _build.LIB


def load(build_if_missing: bool = True):
    """Load libdugma_b200.so (building it in-tree first if it is missing and nvcc exists)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = lib_path()
    if not os.path.exists(path):
        if not build_if_missing:
            raise OSError(f"{path} is missing: build it with `python -m dugma_b200.build`")
        _build.build()
    L = ctypes.CDLL(path)
    for name, (res, args) in EXPORTS.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = L
    return L


def check(rc: int, allow=(OK,)):
    if rc not in allow:
        raise DugmaError(rc, load().dugma_last_error().decode())
    return rc
