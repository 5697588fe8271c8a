"""The seeded generators behind the bench workloads (CPU): deterministic, the documented
shapes, symmetric positive-definite covariances, and ground truth that maps the moving cloud
back onto the fixed one's surface."""
import numpy as np

from dugma_b200 import synth


def test_workload5_2d_curve():
    P = synth.workload5(n=4096)
    Q = synth.workload5(n=4096)
    assert np.array_equal(P.X, Q.X) and np.array_equal(P.Y, Q.Y)          # seeded
    assert P.X.shape == (4096, 2) and P.Y.shape == (4096, 2)
    assert P.X_C.shape == (4096, 2, 2) and P.Y_C.shape == (4096, 2, 2)
    for C in (P.X_C, P.Y_C):
        assert np.allclose(C, np.transpose(C, (0, 2, 1)))
        ev = np.linalg.eigvalsh(C)
        assert np.allclose(ev[:, 0], 0.004 ** 2) and np.allclose(ev[:, 1], 0.01 ** 2)
    assert np.allclose(P.R_G @ P.R_G.T, np.eye(2)) and np.linalg.det(P.R_G) > 0
    # R_G y + t_G lies on the fixed cloud's curve up to the noise: its radius at its angle
    # matches the radius of the nearest fixed point in angle
    Z = P.Y @ P.R_G.T + P.t_G
    az, rz = np.arctan2(Z[:, 1], Z[:, 0]), np.linalg.norm(Z, axis=1)
    ax, rx = np.arctan2(P.X[:, 1], P.X[:, 0]), np.linalg.norm(P.X, axis=1)
    order = np.argsort(ax)
    pos = np.clip(np.searchsorted(ax[order], az), 0, len(ax) - 1)
    assert np.median(np.abs(rz - rx[order][pos])) < 0.02


def test_workload_table():
    assert set(synth.WORKLOADS) == {0, 1, 2, 4, 5}
    P = synth.workload0(n=500)
    assert P.X.shape == (500, 3) and P.X_C.shape == (500, 3, 3)
