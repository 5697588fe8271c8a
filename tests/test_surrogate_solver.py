"""The fmincon stand-in (dugma_minimise_surrogate) on the CPU, against scipy.

Coefficients come from the FP64 oracle's compi at a perturbed pose; the surrogate
Q(dR, dt) = A . b(dR, dt) (energy3D.m:15-16) is minimised over dR in SO(3) by the
library and by scipy (BFGS on the rotation vector); both must reach the same minimum."""
import ctypes

import numpy as np
from scipy.optimize import minimize

from oracle import oracle as orc
from dugma_b200 import _lib, synth
from dugma_b200.monomials import surrogate
from dugma_b200.pose import expmap, rot2d


def _solve(D, A):
    L = _lib.load()
    dR = np.zeros(D * D)
    dt = np.zeros(D)
    q = ctypes.c_double()
    flag = ctypes.c_int()
    rc = L.dugma_minimise_surrogate(D, np.ascontiguousarray(A, np.float64).ctypes.data_as(_lib.dp),
                                    dR.ctypes.data_as(_lib.dp), dt.ctypes.data_as(_lib.dp), ctypes.byref(q),
                                    ctypes.byref(flag))
    assert rc == 0 and flag.value >= 0
    return dR.reshape(D, D).T, dt, q.value


def test_surrogate_minimum_3d_matches_scipy():
    P = synth.workload0(n=300)
    st = orc.State(P.X, P.X_C, P.Y, P.Y_C)
    R = P.R_G @ expmap([0.1, -0.05, 0.08])
    t = P.t_G + 0.02
    sig = st.sigma(R, t)
    A = st.coef(R, t, sig)[:637]
    dR, dt, q = _solve(3, A)
    assert np.allclose(dR @ dR.T, np.eye(3), atol=1e-12) and np.linalg.det(dR) > 0
    assert abs(q - surrogate(3, A, dR, dt)) <= 1e-9 * abs(q)
    f = lambda p: surrogate(3, A, expmap(p[:3]), p[3:]) / abs(A[0])
    res = minimize(f, np.zeros(6), method="BFGS", options={"gtol": 1e-12, "maxiter": 2000})
    q_scipy = res.fun * abs(A[0])
    assert q <= q_scipy + 1e-7 * abs(q_scipy)
    assert np.allclose(np.concatenate([expmap(res.x[:3]).ravel(), res.x[3:]]),
                       np.concatenate([dR.ravel(), dt]), atol=1e-4)


def test_surrogate_minimum_2d_matches_scipy():
    rng = np.random.default_rng(2)
    n = 200
    X = rng.standard_normal((n, 2))
    Y = X @ rot2d(0.2).T + 0.05 + 0.02 * rng.standard_normal((n, 2))
    C = np.tile(np.eye(2) * 0.01, (n, 1, 1))
    st = orc.State(X, C, Y, C)
    A = st.coef(np.eye(2), np.zeros(2), 0.05)[:45]
    dR, dt, q = _solve(2, A)
    f = lambda p: surrogate(2, A, rot2d(p[0]), p[1:]) / abs(A).max()
    res = minimize(f, np.zeros(3), method="BFGS", options={"gtol": 1e-12})
    assert q <= res.fun * abs(A).max() * (1 - 1e-9) + 1e-9 * abs(q) or np.isclose(q, res.fun * abs(A).max(), rtol=1e-7)
    assert np.allclose(dR, rot2d(res.x[0]), atol=1e-5)
