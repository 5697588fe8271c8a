"""ctypes front end of the FP64 CPU oracle (oracle/dugma_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline / reference leg, never by the dugma_b200 package.

Array conventions follow the reference's MEX arguments: X (N, D) float64 point
rows (MATLAB D x N column-major), covariances (N, D, D) per-point blocks,
R (D, D) applied to Y (y' = R y + t).  R is passed to C column-major.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")


def build() -> str:
    path = os.path.join(HERE, "liboracle.so")
    src = [os.path.join(HERE, f) for f in ("dugma_oracle.c", "coef_terms.h")]
    if not os.path.exists(path) or any(os.path.getmtime(s) > os.path.getmtime(path) for s in src):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return path


def lib():
    global _LIB
    if _LIB is None:
        L = ctypes.CDLL(build())
        L.dugma_oracle_prepare.argtypes = [ctypes.c_int, ctypes.c_int, _f64p, _f32p, _f32p]
        L.dugma_oracle_prepare.restype = ctypes.c_int
        L.dugma_oracle_pose.argtypes = [ctypes.c_int, ctypes.c_int, _f32p, _f64p, _f64p, _f64p]
        L.dugma_oracle_energy.argtypes = [ctypes.c_int] * 3 + [_f32p] * 6 + [_f64p, _f64p, ctypes.c_double,
                                                                            ctypes.c_int, ctypes.c_int, _f64p, ctypes.c_void_p]
        L.dugma_oracle_energy_conv.argtypes = [ctypes.c_int] * 3 + [_f32p] * 4 + [_f64p, _f64p, ctypes.c_double,
                                                                                 ctypes.c_int, ctypes.c_int, _f64p, ctypes.c_void_p]
        L.dugma_oracle_nn.argtypes = [ctypes.c_int] * 3 + [_f32p, _f32p, _f64p, _f64p, ctypes.c_int, _i32p, _f32p]
        L.dugma_oracle_sigma.argtypes = [ctypes.c_int, ctypes.c_int, _f32p, ctypes.c_int]
        L.dugma_oracle_sigma.restype = ctypes.c_double
        L.dugma_oracle_coef.argtypes = [ctypes.c_int] * 3 + [_f32p] * 6 + [_f64p, _f64p, ctypes.c_double, _f64p]
        L.dugma_oracle_num_threads.restype = ctypes.c_int
        L.dugma_oracle_set_threads.restype = ctypes.c_int
        L.dugma_oracle_set_threads.argtypes = [ctypes.c_int]
        _LIB = L
    return _LIB


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _cm(R):
    """Column-major flattening of a D x D matrix (MATLAB order)."""
    return np.ascontiguousarray(np.asarray(R, dtype=np.float64).T.reshape(-1))


def prepare(cov: np.ndarray):
    """Reference `init` state for one cloud: (inverse covariances float32 (n,D,D), weights |S|^-1/2 float32 (n,), #neglected)."""
    cov = np.ascontiguousarray(cov, dtype=np.float64)
    n, D = cov.shape[0], cov.shape[1]
    # per-point blocks are column-major in memory: pass the transposed blocks
    cm = np.ascontiguousarray(np.transpose(cov, (0, 2, 1)))
    cinv = np.zeros((n, D, D), np.float32)
    w = np.zeros(n, np.float32)
    bad = lib().dugma_oracle_prepare(D, n, cm.reshape(-1), cinv.reshape(-1), w)
    return np.ascontiguousarray(np.transpose(cinv, (0, 2, 1))), w, bad


class State:
    """FP32 device state produced by the reference's `init` (init.cu:249-348)."""

    def __init__(self, X, X_C, Y, Y_C):
        self.D = X.shape[1]
        self.x = _f32(X)
        self.y = _f32(Y)
        self.xinv, self.wx, self.badx = prepare(X_C)
        self.yinv, self.wy, self.bady = prepare(Y_C)
        self.xcov = _f32(X_C)
        self.ycov = _f32(Y_C)

    @property
    def N(self):
        return self.x.shape[0]

    @property
    def M(self):
        return self.y.shape[0]

    def _cmv(self, a):
        return np.ascontiguousarray(np.transpose(a, (0, 2, 1))).reshape(-1)

    def energy(self, R, t, sig, i0=0, i1=None, with_dx=False):
        """REF energy and pose gradient: (E, g[NR + D], dEdx or None)."""
        i1 = self.N if i1 is None else i1
        out = np.zeros(8)
        dx = np.zeros((i1 - i0, self.D)) if with_dx else None
        lib().dugma_oracle_energy(self.D, self.N, self.M, self.x.reshape(-1), self._cmv(self.xinv), self.wx,
                                  self.y.reshape(-1), self._cmv(self.yinv), self.wy, _cm(R),
                                  np.ascontiguousarray(t, np.float64), float(sig), i0, i1, out,
                                  dx.ctypes.data if with_dx else None)
        ng = 6 if self.D == 3 else 3
        return out[0], out[1:1 + ng].copy(), dx

    def energy_conv(self, R, t, sig, i0=0, i1=None, with_dx=False):
        i1 = self.N if i1 is None else i1
        out = np.zeros(8)
        dx = np.zeros((i1 - i0, self.D)) if with_dx else None
        lib().dugma_oracle_energy_conv(self.D, self.N, self.M, self.x.reshape(-1), self._cmv(self.xcov),
                                       self.y.reshape(-1), self._cmv(self.ycov), _cm(R),
                                       np.ascontiguousarray(t, np.float64), float(sig), i0, i1, out,
                                       dx.ctypes.data if with_dx else None)
        ng = 6 if self.D == 3 else 3
        return out[0], out[1:1 + ng].copy(), dx

    def nn(self, R, t, k=1):
        idx = np.zeros((self.N, k), np.int32)
        d2 = np.zeros((self.N, k), np.float32)
        rc = lib().dugma_oracle_nn(self.D, self.N, self.M, self.x.reshape(-1), self.y.reshape(-1), _cm(R),
                                   np.ascontiguousarray(t, np.float64), k, idx.reshape(-1), d2.reshape(-1))
        if rc:
            raise ValueError("bad k")
        return idx, d2

    def sigma(self, R, t, quantised=True):
        _, d2 = self.nn(R, t, 1)
        return lib().dugma_oracle_sigma(self.D, self.N, np.ascontiguousarray(d2[:, 0]), 1 if quantised else 0)

    def coef(self, R, t, sig):
        out = np.zeros(640)
        lib().dugma_oracle_coef(self.D, self.N, self.M, self.x.reshape(-1), self._cmv(self.xinv), self.wx,
                                self.y.reshape(-1), self._cmv(self.yinv), self.wy, _cm(R),
                                np.ascontiguousarray(t, np.float64), float(sig), out)
        return out


def num_threads() -> int:
    return lib().dugma_oracle_num_threads()


def use_all_cores() -> int:
    """Run the oracle on every host core (launchers may have set OMP_NUM_THREADS=1)."""
    import os
    n = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    return lib().dugma_oracle_set_threads(n)


# ---------------------------------------------------------------------------
# Pure-numpy restatement (small cases only): an independent second oracle for
# the REF energy and the per-pair quadratic q used to pin the C oracle.
# ---------------------------------------------------------------------------
def np_derived(st: State, R, t, sig):
    s = 1.0 / sig
    D = st.D
    yp = st.y.astype(np.float64) @ np.asarray(R).T + np.asarray(t)
    A = st.yinv.astype(np.float64) * s
    A = 0.5 * (A + np.transpose(A, (0, 2, 1)))
    Cp = np.einsum("ab,jbc,dc->jad", R, A, R)
    B = st.xinv.astype(np.float64) * s
    B = 0.5 * (B + np.transpose(B, (0, 2, 1)))
    w = st.wx.astype(np.float64) * s ** (D / 2)
    v = st.wy.astype(np.float64) * s ** (D / 2)
    return yp, Cp, B, w, v


def np_pair_weights(st: State, R, t, sig):
    """P_ij (N, M) in FP64 (compi.cu:753-772)."""
    yp, Cp, B, w, v = np_derived(st, R, t, sig)
    x = st.x.astype(np.float64)
    d = x[:, None, :] - yp[None, :, :]
    m1 = np.einsum("ija,jab,ijb->ij", d, Cp, d)
    m2 = np.einsum("ija,iab,ijb->ij", d, B, d)
    return w[:, None] * v[None, :] * (np.exp(-0.5 * m1) + np.exp(-0.5 * m2))


def np_surrogate_direct(st: State, R, t, sig, dR, dt):
    """sum_ij P_ij q_ij(dR, dt) evaluated directly (the identity behind the coefficients)."""
    yp, Cp, B, w, v = np_derived(st, R, t, sig)
    P = np_pair_weights(st, R, t, sig)
    x = st.x.astype(np.float64)
    e = x[:, None, :] - (yp @ np.asarray(dR).T)[None, :, :] - np.asarray(dt)
    M1 = np.einsum("ab,jbc,dc->jad", dR, Cp, dR)
    q = np.einsum("ija,jab,ijb->ij", e, M1, e) + np.einsum("ija,iab,ijb->ij", e, B, e)
    return float(np.sum(P * q))


def monomial_values(D, dR, dt, exps):
    """b_k(dR, dt) for the exponent table (variables t..., then r11 r12 r13 r21 ... row-major)."""
    if D == 3:
        v = np.concatenate([np.asarray(dt, float), np.asarray(dR, float).reshape(-1)])
    else:
        v = np.array([dt[0], dt[1], dR[0][0], dR[1][0]], float)
    return np.prod(v[None, :] ** np.asarray(exps, float), axis=1)
