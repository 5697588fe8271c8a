"""ctypes harness for the reference's own CUDA plugins built by oracle/ref_build.py.

Test infrastructure only: used by tests/golden/make_golden.py (run on a GPU) to record the
reference's outputs, and by bench.py to time the reference kernels on the same GPU.
It calls the reference's C++ entry points by their mangled names, exactly as the MEX
gateways do (init.cpp:65, update_sig.cpp:45, compi.cpp:45).  fr_m is never called:
it ends with cudaDeviceReset (fr_m.cu:27), which would tear down the caller's context.

compi's kernel synchronises inside `if (ix < N && iy < M)` (compi.cu:794, 803), which
is only well defined when every thread of a 32 x 32 block takes that branch, i.e. when
N and M are multiples of 32; `compi` below refuses other sizes.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_dp = ctypes.POINTER(ctypes.c_double)
PtrArray = ctypes.c_void_p * 6


def available() -> bool:
    return all(os.path.exists(os.path.join(HERE, "_ref", f"libref_{n}.so")) for n in ("init", "update_sig", "compi"))


_libs = {}


def _lib(name):
    if name not in _libs:
        _libs[name] = ctypes.CDLL(os.path.join(HERE, "_ref", f"libref_{name}.so"))
    return _libs[name]


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def init(X, X_C, Y, Y_C):
    """Reference init: returns the six device pointers (the reference prints them)."""
    X, Y = _d(X), _d(Y)
    N, D = X.shape
    M = Y.shape[0]
    XC = _d(np.transpose(X_C, (0, 2, 1)))
    YC = _d(np.transpose(Y_C, (0, 2, 1)))
    f = getattr(_lib("init"), "_Z4initPdS_S_S_S_iiiPPf")
    f.restype = None
    ptr = PtrArray()
    coef = ctypes.c_double(0)
    f(X.ctypes.data_as(_dp), XC.ctypes.data_as(_dp), Y.ctypes.data_as(_dp), YC.ctypes.data_as(_dp),
      ctypes.byref(coef), N, M, D, ptr)
    assert coef.value == 1.0
    return ptr


def update_sig(ptr, R, t, N, M, D) -> float:
    f = getattr(_lib("update_sig"), "_Z3cpdPPfPdS1_S1_S1_S1_S_")
    f.restype = None
    sig = ctypes.c_float(0)
    n, m, d = ctypes.c_double(N), ctypes.c_double(M), ctypes.c_double(D)
    f(ptr, _d(np.asarray(R).T).ctypes.data_as(_dp), _d(t).ctypes.data_as(_dp), ctypes.byref(n), ctypes.byref(m),
      ctypes.byref(d), ctypes.byref(sig))
    return float(sig.value)


def compi(ptr, R, t, N, M, D, sig) -> np.ndarray:
    if N % 32 or M % 32:
        raise ValueError("the reference compi kernel is only well defined for N, M multiples of 32")
    f = getattr(_lib("compi"), "_Z3cpdPPfPdS1_S1_S1_S1_S1_S1_")
    f.restype = None
    out = np.zeros(640)
    n, m, d, s = ctypes.c_double(N), ctypes.c_double(M), ctypes.c_double(D), ctypes.c_double(sig)
    f(ptr, _d(np.asarray(R).T).ctypes.data_as(_dp), _d(t).ctypes.data_as(_dp), ctypes.byref(n), ctypes.byref(m),
      ctypes.byref(d), ctypes.byref(s), out.ctypes.data_as(_dp))
    return out
