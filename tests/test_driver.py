"""Registration driver (DUGMA.m's loop, quasi-Newton in place of fmincon) on the GPU.

End-to-end checks against the seeded ground truth, in the error metric of
main_simulation.m:63-64 (||I - R R_G^-1||_F) plus the geodesic angle."""
import numpy as np
import pytest

from dugma_b200 import api, synth
from dugma_b200.pose import expmap, rotation_error_deg

pytestmark = pytest.mark.gpu


def _errors(R, t, R_G, t_G):
    return rotation_error_deg(R, R_G), float(np.linalg.norm(np.eye(len(R)) - R @ np.linalg.inv(R_G))), \
        float(np.linalg.norm(t - t_G))


@pytest.mark.parametrize("mode", [0, 1])
def test_register_sphere_from_identity(mode):
    P = synth.workload0()
    R, t, stats = api.DUGMA(P.X, P.Y, P.X_C, P.Y_C, np.eye(3), np.zeros(3), Max_Iteration=100, mode=mode)
    deg, fro, terr = _errors(R, t, P.R_G, P.t_G)
    print(f"mode {mode}: {deg:.3f} deg, |I - R R_G^-1|_F {fro:.4f}, |t - t_G| {terr:.4f}, iterations {stats[0]:.0f},"
          f" sigma {stats[1]:.3e}, {stats[4]:.2f} s")
    assert deg < 2.0 and terr < 0.05


def test_register_2d():
    rng = np.random.default_rng(1)
    n = 600
    th = rng.uniform(0, 2 * np.pi, n)
    S = np.stack([np.cos(th) * (1 + 0.3 * np.sin(3 * th)), np.sin(th) * (1 + 0.3 * np.sin(3 * th))], 1)
    X = S + 0.005 * rng.standard_normal(S.shape)
    a = 0.4
    Rm = np.array([[np.cos(a), -np.sin(a)], [np.sin(a), np.cos(a)]])
    Y = (S[rng.permutation(n)] @ Rm.T) + np.array([0.2, -0.1])
    XC = np.tile(np.eye(2) * 1e-4, (n, 1, 1))
    YC = np.tile(np.eye(2) * 1e-4, (n, 1, 1))
    R, t, stats = api.DUGMA(X, Y, XC, YC, np.eye(2), np.zeros(2), Max_Iteration=100)
    R_G = Rm.T
    t_G = -Rm.T @ np.array([0.2, -0.1])
    ang = abs(np.degrees(np.arctan2(R[1, 0], R[0, 0]) - np.arctan2(R_G[1, 0], R_G[0, 0])))
    print(f"2D: {ang:.3f} deg, |t - t_G| {np.linalg.norm(t - t_G):.4f}, iterations {stats[0]:.0f}")
    assert ang < 1.0 and np.linalg.norm(t - t_G) < 0.02
