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


def test_batch_workload3_as_configured():
    """The configured batch: 256 problems with N, M uniform in [500, 8000], 32 rotations of a
    uniform SO(3) grid each, all evaluated in one persistent launch.  Every result is finite; 8
    sampled (problem, pose) pairs match the single-problem adjoint and the FP64 oracle (energy
    1e-6, pose gradient 1e-5 relative); the autotuner times every tile shape and the shape it
    keeps gives the same results within the same tolerances."""
    probs = synth.workload3()
    grid = synth.so3_grid(synth.rng_for(3, 1), 32)
    P, Q = len(probs), len(grid)
    assert (P, Q) == (256, 32)
    sig = np.zeros((P, Q))
    for p, pr in enumerate(probs):
        _, h = api.init(pr.X, pr.X_C, pr.Y, pr.Y_C)
        sig[p, :] = api.update_sig(h, np.eye(3), pr.t_G)
        api.fr_m(h)
    R = np.array([[gq @ pr.R_G for gq in grid] for pr in probs])
    t = np.array([[pr.t_G for _ in grid] for pr in probs])
    b = api.Batch([(pr.X, pr.X_C, pr.Y, pr.Y_C) for pr in probs])
    try:
        E, g = b.energy_grad(R, t, sig)
        assert np.all(np.isfinite(E)) and np.all(np.isfinite(g)) and np.all(E > 0)
        rng = np.random.default_rng(33)
        picks = [(int(p), int(q)) for p, q in zip(rng.choice(P, 8, replace=False), rng.integers(0, Q, 8))]
        for p, q in picks:
            pr = probs[p]
            _, h = api.init(pr.X, pr.X_C, pr.Y, pr.Y_C)
            try:
                Es, gs, _ = api.energy_grad(h, R[p, q], t[p, q], sig[p, q])
            finally:
                api.fr_m(h)
            Eo, go, _ = orc.State(pr.X, pr.X_C, pr.Y, pr.Y_C).energy(R[p, q], t[p, q], sig[p, q])
            for Eref, gref in ((Es, gs), (Eo, go)):
                assert abs(E[p, q] - Eref) <= 1e-6 * abs(Eref), (p, q, E[p, q], Eref)
                assert np.linalg.norm(g[p, q] - gref) <= 1e-5 * np.linalg.norm(gref), (p, q)
        rep = b.autotune(R, t, sig)
        assert rep.count("ms") == len(api.Batch.shapes()), rep
        assert b.get_shape() in api.Batch.shapes()
        E2, g2 = b.energy_grad(R, t, sig)
        assert np.all(np.abs(E2 - E) <= 1e-6 * np.abs(E))
        assert np.all(np.linalg.norm(g2 - g, axis=-1) <= 1e-5 * np.linalg.norm(g, axis=-1))
    finally:
        b.close()


def test_batch_shapes_give_the_same_results():
    """Every compiled batch tile shape on the small uneven batch, against the default shape."""
    probs = _batch(seed=3)
    P, Q = len(probs), 3
    rng = np.random.default_rng(5)
    R = np.array([[expmap(rng.standard_normal(3) * 0.3) for _ in range(Q)] for _ in range(P)])
    t = rng.standard_normal((P, Q, 3)) * 0.05
    sig = rng.uniform(0.005, 0.05, (P, Q))
    b = api.Batch(probs)
    try:
        shapes = api.Batch.shapes()
        assert b.get_shape() == shapes[0]
        E0, g0 = b.energy_grad(R, t, sig)
        for sh in shapes[1:]:
            b.set_shape(sh)
            E, g = b.energy_grad(R, t, sig)
            assert np.all(np.abs(E - E0) <= 1e-6 * np.abs(E0)), sh
            assert np.all(np.linalg.norm(g - g0, axis=-1) <= 1e-5 * np.linalg.norm(g0, axis=-1)), sh
        b.timing(1)
        b.energy_grad(R, t, sig)
        b.energy_grad(R, t, sig)
        ms, n = b.timing(2)
        assert n == 2 and ms > 0
    finally:
        b.close()
