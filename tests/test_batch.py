"""Batched evaluation (uneven problems x multistart poses, one persistent launch + graph replay)
against the single-problem adjoint and the FP64 oracle."""
import numpy as np
import pytest

from oracle import oracle as orc
from dugma_b200 import api, synth
from dugma_b200.pose import expmap

pytestmark = pytest.mark.gpu


def _batch(seed=0, sizes=((300, 800), (1500, 257), (64, 64), (1025, 1000), (700, 1300))):
    rng = np.random.default_rng(seed)
    probs = []
    for (n, m) in sizes:
        X = synth.bumpy_sphere(rng, n)
        S = synth.bumpy_sphere(rng, m)
        Y = S @ expmap(rng.standard_normal(3) * 0.2).T + 0.05
        probs.append((X, synth._sensor_diag_cov(X), Y, synth._sensor_diag_cov(Y)))
    return probs


def test_batch_matches_single_problem_and_oracle():
    probs = _batch()
    P, Q = len(probs), 4
    rng = np.random.default_rng(1)
    R = np.array([[expmap(rng.standard_normal(3) * 0.3) for _ in range(Q)] for _ in range(P)])
    t = rng.standard_normal((P, Q, 3)) * 0.05
    sig = rng.uniform(0.005, 0.05, (P, Q))
    b = api.Batch(probs)
    try:
        E, g = b.energy_grad(R, t, sig)
        E2, g2 = b.energy_grad(R, t, sig)          # graph replay
        assert np.array_equal(E, E2) and np.array_equal(g, g2)
        for p, (X, XC, Y, YC) in enumerate(probs):
            _, h = api.init(X, XC, Y, YC)
            try:
                for q in range(Q):
                    Es, gs, _ = api.energy_grad(h, R[p, q], t[p, q], sig[p, q])
                    assert abs(E[p, q] - Es) <= 1e-6 * abs(Es), (p, q)
                    assert np.linalg.norm(g[p, q] - gs) <= 1e-5 * np.linalg.norm(gs), (p, q)
            finally:
                api.fr_m(h)
        st = orc.State(*probs[1])
        Eo, go, _ = st.energy(R[1, 2], t[1, 2], sig[1, 2])
        assert abs(E[1, 2] - Eo) <= 1e-6 * Eo
        assert np.linalg.norm(g[1, 2] - go) <= 1e-5 * np.linalg.norm(go)
        # new poses through the same graph
        E3, g3 = b.energy_grad(R[:, ::-1], t[:, ::-1], sig[:, ::-1])
        assert np.allclose(E3, E[:, ::-1], rtol=1e-12, atol=0)
    finally:
        b.close()
