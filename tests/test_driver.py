"""Registration driver (DUGMA.m's loop, quasi-Newton in place of fmincon) on the GPU.

The data follow the reference's simulation (main_simulation.m:12-51,
noise_and_sampling3D.m:49-57): diagonal "uncertainty" covariances exp(3.4657 |noise|)
(>= 1, i.e. wide relative to the normalised cloud) and a rotation of about 10 degrees.
Errors use the metric of main_simulation.m:63-64 plus the geodesic angle."""
import numpy as np
import pytest

from dugma_b200 import api, synth
from dugma_b200.pose import expmap, rot2d, rotation_error_deg

pytestmark = pytest.mark.gpu


def _uncertainty_covs(rng, n, D):
    v = np.exp(3.4657 * np.abs(0.05 * rng.standard_normal((n, D))))
    return np.einsum("na,ab->nab", v, np.eye(D))


def _problem3d(seed=0, n=1000):
    rng = np.random.default_rng(seed)
    S = synth.workload0(n=n).X
    Rm = expmap(np.radians([6.0, -5.0, 6.0]))
    tm = np.array([0.05, -0.03, 0.04])
    Y = S[rng.permutation(n)] @ Rm.T + tm + 0.005 * rng.standard_normal(S.shape)
    return S, _uncertainty_covs(rng, n, 3), Y, _uncertainty_covs(rng, n, 3), Rm.T, -Rm.T @ tm


@pytest.mark.parametrize("mode", [0, 1])
def test_register_3d(mode):
    X, XC, Y, YC, R_G, t_G = _problem3d()
    R, t, stats = api.DUGMA(X, Y, XC, YC, np.eye(3), np.zeros(3), Max_Iteration=300, mode=mode)
    deg = rotation_error_deg(R, R_G)
    fro = float(np.linalg.norm(np.eye(3) - R @ np.linalg.inv(R_G)))
    terr = float(np.linalg.norm(t - t_G))
    print(f"mode {mode}: {deg:.4f} deg, |I - R R_G^-1|_F {fro:.5f}, |t - t_G| {terr:.5f}, "
          f"iterations {stats[0]:.0f}, sigma {stats[1]:.3e}, {stats[4]:.2f} s")
    assert deg < 0.5 and terr < 0.01


def test_register_2d():
    rng = np.random.default_rng(1)
    n = 600
    th = rng.uniform(0, 2 * np.pi, n)
    S = np.stack([np.cos(th) * (1 + 0.3 * np.sin(3 * th)), np.sin(th) * (1 + 0.3 * np.sin(3 * th))], 1)
    a = np.radians(10.0)
    Rm = rot2d(a)
    tm = np.array([0.05, -0.04])
    Y = S[rng.permutation(n)] @ Rm.T + tm + 0.005 * rng.standard_normal(S.shape)
    R, t, stats = api.DUGMA(S, Y, _uncertainty_covs(rng, n, 2), _uncertainty_covs(rng, n, 2), np.eye(2),
                            np.zeros(2), Max_Iteration=300)
    R_G, t_G = Rm.T, -Rm.T @ tm
    ang = abs(np.degrees(np.arctan2(R[1, 0], R[0, 0]) - np.arctan2(R_G[1, 0], R_G[0, 0])))
    print(f"2D: {ang:.4f} deg, |t - t_G| {np.linalg.norm(t - t_G):.5f}, iterations {stats[0]:.0f}")
    assert ang < 0.5 and np.linalg.norm(t - t_G) < 0.01


def test_register_degenerate_input_is_an_error_not_a_crash():
    """One point per cloud has no scale (normalize.m divides by the RMS radius): a status, not an abort."""
    from dugma_b200._lib import DugmaError
    C = np.eye(3)[None]
    with pytest.raises(DugmaError):
        api.DUGMA(np.ones((1, 3)), -np.ones((1, 3)), C, C, np.eye(3), np.zeros(3), Max_Iteration=5)
