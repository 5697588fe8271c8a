"""Python mirror of the reference's plugin interface over the C ABI.

The reference's MATLAB code calls four MEX plugins (DUGMA.m:44-126):

    [Success, ad0..ad5] = init(X, X_C, Y, Y_C)                    init.cpp:36-83
    [sig, ad0..ad5]     = update_sig(ad0..ad5, R, t, N, M, D)     update_sig.cpp:8-65
    [A, ad0..ad5]       = compi(ad0..ad5, R, t, N, M, D, sig)     compi.cpp:8-73
    Success             = fr_m(ad0..ad5)                          fr_m.cpp:8-34

This module offers the same four calls (`init`, `update_sig`, `compi`, `fr_m`)
with the same argument meaning, and `DUGMA(...)` for the whole registration
loop.  Arrays follow numpy conventions: X is (N, D) (one point per row, the
memory layout of MATLAB's D x N), X_C is (N, D, D) with X_C[p] point p's
covariance, R is a (D, D) matrix with y' = R y + t.  Device handles are a
`Handles` object (the six pointers ad0..ad5).  Errors raise DugmaError
instead of exiting the process.
"""
from __future__ import annotations

import ctypes
import warnings

import numpy as np

from . import _lib
from ._lib import DugmaError, check

_dp = _lib.dp


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _ptr(a):
    return a.ctypes.data_as(_dp)


def _cm(R):
    """(D, D) matrix -> MATLAB column-major doubles."""
    return _d(np.asarray(R, dtype=np.float64).T)


def _blocks(C):
    """(n, D, D) covariances -> MATLAB D x (D n) column-major per-point blocks."""
    return _d(np.transpose(np.asarray(C, dtype=np.float64), (0, 2, 1)))


class Handles:
    """The six device pointers ad0..ad5 returned by init (d_X, d_X_C^-1, d_Y, d_Y_C^-1, det_X, det_Y)."""

    def __init__(self, N: int, M: int, D: int):
        self.arr = _lib.PtrArray()
        self.N, self.M, self.D = N, M, D
        self.alive = True

    @property
    def ptrs(self):
        return [self.arr[k] for k in range(6)]


def init(X, X_C, Y, Y_C):
    """Upload both clouds, invert the covariances; returns (Success = 1.0, Handles).

    Covariances with det <= 0 are neglected as in the reference (a warning is issued)."""
    X, Y = _d(X), _d(Y)
    N, D = X.shape
    M = Y.shape[0]
    if Y.shape[1] != D or np.shape(X_C) != (N, D, D) or np.shape(Y_C) != (M, D, D):
        raise DugmaError(_lib.ERR_ARG, "shapes must be X (N,D), Y (M,D), X_C (N,D,D), Y_C (M,D,D)")
    XC, YC = _blocks(X_C), _blocks(Y_C)
    h = Handles(N, M, D)
    coef = ctypes.c_double(0)
    L = _lib.load()
    rc = L.dugma_init(_ptr(X), _ptr(XC), _ptr(Y), _ptr(YC), ctypes.byref(coef), N, M, D, h.arr)
    check(rc, allow=(_lib.OK, _lib.ERR_NONPD))
    if rc == _lib.ERR_NONPD:
        warnings.warn(L.dugma_last_error().decode())
    return coef.value, h


def _nmd(h: Handles, N=None, M=None, D=None):
    N = h.N if N is None else N
    M = h.M if M is None else M
    D = h.D if D is None else D
    return (ctypes.c_double(N), ctypes.c_double(M), ctypes.c_double(D))


def update_sig(h: Handles, R, t, N=None, M=None, D=None) -> float:
    """sig = mean_i min_j |x_i - (R y_j + t)|^2 / D with the reference's 1e-6 quantisation."""
    n, m, d = _nmd(h, N, M, D)
    sig = ctypes.c_float(0)
    check(_lib.load().dugma_update_sig(h.arr, _ptr(_cm(R)), _ptr(_d(t)), ctypes.byref(n), ctypes.byref(m),
                                       ctypes.byref(d), ctypes.byref(sig)))
    return float(sig.value)


def compi(h: Handles, R, t, N=None, M=None, D=None, sig=None) -> np.ndarray:
    """The 637 (3D) / 45 (2D) surrogate coefficients in the energy3D.m / energy2D.m order."""
    n, m, d = _nmd(h, N, M, D)
    s = ctypes.c_double(sig)
    out = np.zeros(640)
    check(_lib.load().dugma_compi(h.arr, _ptr(_cm(R)), _ptr(_d(t)), ctypes.byref(n), ctypes.byref(m),
                                  ctypes.byref(d), ctypes.byref(s), _ptr(out)))
    return out[: 637 if h.D == 3 else 45].copy()


def compi_range(h: Handles, R, t, sig, i0, i1, j0, j1) -> np.ndarray:
    """Partial coefficients: source-side terms of source rows [i0, i1) plus target-side terms of
    target rows [j0, j1); partials over partitions of both ranges sum to compi's."""
    out = np.zeros(640)
    check(_lib.load().dugma_compi_range(h.arr, _ptr(_cm(R)), _ptr(_d(t)), float(sig), int(i0), int(i1), int(j0),
                                        int(j1), _ptr(out)))
    return out[: 637 if h.D == 3 else 45].copy()


def fr_m(h: Handles) -> float:
    check(_lib.load().dugma_fr_m(h.arr))
    h.alive = False
    return 1.0


# ---------------------------------------------------------------------------
# energy / adjoint / nearest neighbours
# ---------------------------------------------------------------------------
def ngrad(D: int) -> int:
    return 6 if D == 3 else 3


def energy(h: Handles, R, t, sig, model=_lib.MODEL_REF) -> float:
    E = ctypes.c_double(0)
    check(_lib.load().dugma_energy(h.arr, _ptr(_cm(R)), _ptr(_d(t)), float(sig), model, ctypes.byref(E)))
    return E.value


def energy_grad(h: Handles, R, t, sig, model=_lib.MODEL_REF, with_dx=False):
    """(E, g, dEdx): g = [dE/domega, dE/dt] for R <- exp([omega]x) R; dEdx (N, D) if with_dx."""
    E = ctypes.c_double(0)
    g = np.zeros(ngrad(h.D))
    dx = np.zeros((h.N, h.D)) if with_dx else None
    check(_lib.load().dugma_energy_grad(h.arr, _ptr(_cm(R)), _ptr(_d(t)), float(sig), model, ctypes.byref(E),
                                        _ptr(g), _ptr(dx) if with_dx else None))
    return E.value, g, dx


def energy_grad_range(h: Handles, R, t, sig, i0, i1, model=_lib.MODEL_REF):
    E = ctypes.c_double(0)
    g = np.zeros(ngrad(h.D))
    check(_lib.load().dugma_energy_grad_range(h.arr, _ptr(_cm(R)), _ptr(_d(t)), float(sig), model, int(i0),
                                              int(i1), ctypes.byref(E), _ptr(g)))
    return E.value, g


def energy_fd_grad(h: Handles, R, t, sig, step=1e-4, model=_lib.MODEL_REF):
    """The plain form: E and central finite differences (1 + 2 NG energy evaluations)."""
    E = ctypes.c_double(0)
    g = np.zeros(ngrad(h.D))
    check(_lib.load().dugma_energy_fd_grad(h.arr, _ptr(_cm(R)), _ptr(_d(t)), float(sig), model, float(step),
                                           ctypes.byref(E), _ptr(g)))
    return E.value, g


def nn(h: Handles, R, t, k=1):
    idx = np.zeros((h.N, k), np.int32)
    d2 = np.zeros((h.N, k), np.float32)
    check(_lib.load().dugma_nn(h.arr, _ptr(_cm(R)), _ptr(_d(t)), int(k),
                               idx.ctypes.data_as(_lib.ip), d2.ctypes.data_as(_lib.fp)))
    return idx, d2


def sigma(h: Handles, R, t) -> float:
    s = ctypes.c_double(0)
    check(_lib.load().dugma_sigma(h.arr, _ptr(_cm(R)), _ptr(_d(t)), ctypes.byref(s)))
    return s.value


def sigma_range(h: Handles, R, t, i0, i1) -> np.ndarray:
    """Partial sums behind sigma over source rows [i0, i1): (sum d2min, sum of quantised terms)."""
    out = np.zeros(2)
    check(_lib.load().dugma_sigma_range(h.arr, _ptr(_cm(R)), _ptr(_d(t)), int(i0), int(i1), _ptr(out)))
    return out


def autotune(h: Handles, what=0, model=_lib.MODEL_REF) -> str:
    buf = ctypes.create_string_buffer(1024)
    check(_lib.load().dugma_autotune(h.arr, int(what), int(model), buf, 1024))
    return buf.value.decode()


def knn_covariance(points, k=8, lo=1e-6, hi=1e-2):
    """Per-point covariance from the k nearest other points (GPU), eigenvalues clamped to [lo, hi]."""
    P = _d(points)
    n, D = P.shape
    out = np.zeros((n, D, D))
    check(_lib.load().dugma_knn_covariance(_ptr(P), n, D, int(k), float(lo), float(hi), _ptr(out)))
    return np.ascontiguousarray(np.transpose(out, (0, 2, 1)))


def shapes(what=0):
    """Compiled kernel shapes for `what` (0 adjoint, 1 energy, 2 nearest neighbour, 3 CONV adjoint,
    4 CONV energy): (ipt, nt, tj, pack)."""
    buf = (ctypes.c_int * 256)()
    n = _lib.load().dugma_shapes(int(what), buf, 64)
    if n < 0:
        check(-n)
    return [tuple(buf[4 * k:4 * k + 4]) for k in range(n)]


def get_shape(h: Handles, what) -> tuple:
    """The kernel shape (ipt, nt, tj, pack) this context uses for `what`."""
    buf = (ctypes.c_int * 4)()
    check(_lib.load().dugma_get_shape(h.arr, int(what), buf))
    return tuple(buf)


def set_shape(h: Handles, what, shape):
    check(_lib.load().dugma_set_shape(h.arr, int(what), *[int(v) for v in shape]))


class Batch:
    """Many registration problems (uneven sizes) evaluated together: one persistent launch
    per evaluation over every (problem, pose) pair, replayed as a CUDA graph after the first."""

    def __init__(self, problems):
        """problems: sequence of (X, X_C, Y, Y_C) in the layout of init."""
        D = np.shape(problems[0][0])[1]
        self.D = D
        self._keep = []
        arrs = []
        for (X, XC, Y, YC) in problems:
            a = (_d(X), _blocks(XC), _d(Y), _blocks(YC))
            self._keep.append(a)
            arrs.append(a)
        P = len(arrs)
        self.P = P
        N = (ctypes.c_int * P)(*[a[0].shape[0] for a in arrs])
        M = (ctypes.c_int * P)(*[a[2].shape[0] for a in arrs])
        ptr = lambda k: (_dp * P)(*[_ptr(a[k]) for a in arrs])
        self.b = ctypes.c_void_p()
        check(_lib.load().dugma_batch_create(P, D, N, M, ptr(0), ptr(1), ptr(2), ptr(3), ctypes.byref(self.b)))

    def _poses(self, R, t, sig):
        R, t, sig = np.asarray(R, float), np.asarray(t, float), np.asarray(sig, float)
        P, Q = sig.shape
        rec = np.zeros((P, Q, 13))
        rec[:, :, : self.D * self.D] = np.transpose(R, (0, 1, 3, 2)).reshape(P, Q, -1)
        rec[:, :, 9:9 + self.D] = t
        rec[:, :, 12] = sig
        return _d(rec), Q

    def energy_grad(self, R, t, sig):
        """R (P, Q, D, D), t (P, Q, D), sig (P, Q) -> E (P, Q), g (P, Q, NG)."""
        rec, Q = self._poses(R, t, sig)
        ng = ngrad(self.D)
        out = np.zeros((self.P, Q, 1 + ng))
        check(_lib.load().dugma_batch_energy_grad(self.b, Q, _ptr(rec), 0, _ptr(out)))
        return out[:, :, 0].copy(), out[:, :, 1:].copy()

    def autotune(self, R, t, sig) -> str:
        """Times every batch tile shape on these poses and keeps the fastest; returns the report."""
        rec, Q = self._poses(R, t, sig)
        buf = ctypes.create_string_buffer(2048)
        check(_lib.load().dugma_batch_autotune(self.b, Q, _ptr(rec), buf, len(buf)))
        return buf.value.decode()

    def set_shape(self, shape):
        check(_lib.load().dugma_batch_set_shape(self.b, *[int(v) for v in shape]))

    def get_shape(self):
        s = (ctypes.c_int * 4)()
        check(_lib.load().dugma_batch_get_shape(self.b, s))
        return tuple(s)

    def timing(self, mode):
        """mode 1 start, 0 stop, 2 -> (total device ms, evaluations) since mode 1."""
        ms, n = ctypes.c_double(0), ctypes.c_int(0)
        check(_lib.load().dugma_batch_timing(self.b, int(mode), ctypes.byref(ms), ctypes.byref(n)))
        return ms.value, n.value

    @staticmethod
    def shapes():
        n = _lib.load().dugma_batch_shapes(None, 0)
        s = (ctypes.c_int * (4 * n))()
        _lib.load().dugma_batch_shapes(s, n)
        return [tuple(s[4 * k:4 * k + 4]) for k in range(n)]

    def close(self):
        if self.b:
            check(_lib.load().dugma_batch_destroy(self.b))
            self.b = ctypes.c_void_p()


class Graph:
    """A captured energy+gradient evaluation, replayed per pose."""

    def __init__(self, h: Handles, model=_lib.MODEL_REF):
        self.h = h
        self.g = ctypes.c_void_p()
        check(_lib.load().dugma_graph_create(h.arr, int(model), ctypes.byref(self.g)))

    def __call__(self, R, t, sig):
        E = ctypes.c_double(0)
        g = np.zeros(ngrad(self.h.D))
        check(_lib.load().dugma_graph_eval(self.g, _ptr(_cm(R)), _ptr(_d(t)), float(sig), ctypes.byref(E), _ptr(g)))
        return E.value, g

    def close(self):
        if self.g:
            check(_lib.load().dugma_graph_destroy(self.g))
            self.g = ctypes.c_void_p()


class EMGraph:
    """update_sig at a pose followed by compi at that pose and sigma, as one captured graph."""

    def __init__(self, h: Handles):
        self.h = h
        self.g = ctypes.c_void_p()
        check(_lib.load().dugma_em_graph_create(h.arr, ctypes.byref(self.g)))

    def __call__(self, R, t):
        """-> (sigma as update_sig returns it, the 637 / 45 coefficients as compi returns them)."""
        sig = ctypes.c_float(0)
        A = np.zeros(640)
        check(_lib.load().dugma_em_step(self.g, _ptr(_cm(R)), _ptr(_d(t)), ctypes.byref(sig), _ptr(A)))
        return float(sig.value), A[:637 if self.h.D == 3 else 45].copy()

    def close(self):
        if self.g:
            check(_lib.load().dugma_em_graph_destroy(self.g))
            self.g = ctypes.c_void_p()


def DUGMA(X, Y, X_C, Y_C, R0, t0, Max_Iteration=300, accuracy_rotation=1e-4, accuracy_translation=1e-8,
          accuracy_sig=1e-8, mode=_lib.DRIVE_REFERENCE):
    """The registration loop of DUGMA.m:19-137 (fmincon replaced by a quasi-Newton solver).

    Returns (R, t, stats) with R @ y + t ~ x in the input coordinates."""
    X, Y = _d(X), _d(Y)
    N, D = X.shape
    M = Y.shape[0]
    R = np.zeros(D * D)
    t = np.zeros(D)
    stats = np.zeros(8)
    check(_lib.load().dugma_register(_ptr(X), _ptr(_blocks(X_C)), _ptr(Y), _ptr(_blocks(Y_C)), N, M, D,
                                     _ptr(_cm(R0)), _ptr(_d(t0)), int(Max_Iteration), float(accuracy_rotation),
                                     float(accuracy_translation), float(accuracy_sig), int(mode), _ptr(R), _ptr(t),
                                     _ptr(stats)))
    return R.reshape(D, D).T.copy(), t, stats
