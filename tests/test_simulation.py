"""The reference's simulation protocol on its own models.

CPU: the seeded generator (synth.simulation, restating produce_point_cloud.m, add_outliers.m,
get_radius.m, noise_and_sampling2D.m and noise_and_sampling3D.m) on the fixture
tests/golden/sim_models.npz (the reference's 2D_SHAPE_MODEL and 2D_Fish_MODEL/dataset2D_200
contours and its 3D_SHAPE surface, written by tests/golden/make_sim_models.py): without noise,
outliers or occlusion the ground truth maps Y exactly onto the model; covariances are
axis-aligned in X's frame and rotated in Y's; the draws stay in the protocol's ranges.
GPU: main_simulation.m's registration (identity start, 700 iterations, tolerances 1e-4 / 1e-8 /
1e-9) of 20 problems per model set with the reference's loop (mode 0): a median under 1 degree
and at least 85 % of the problems within 2 degrees of the ground truth.  The misses are the
problems whose random outliers and occlusion move the energy's maximum away from the truth.
"""
import math
import os

import numpy as np
import pytest

from dugma_b200 import synth

FIX = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "sim_models.npz")


def _models():
    return np.load(FIX)


def _deg(R):
    if R.shape[0] == 2:
        return abs(math.degrees(math.atan2(R[1, 0], R[0, 0])))
    return math.degrees(math.acos(max(-1.0, min(1.0, (np.trace(R) - 1) / 2))))


def test_fixture_holds_the_reference_models():
    f = _models()
    assert sorted(f.files) == sorted([f"S{k}" for k in range(1, 101)] + [f"F{k}" for k in range(1, 101)] + ["T1"])
    sizes_s = [f[f"S{k}"].shape[0] for k in range(1, 101)]
    sizes_f = [f[f"F{k}"].shape[0] for k in range(1, 101)]
    assert min(sizes_s) == 206 and max(sizes_s) == 532
    assert min(sizes_f) == 162 and max(sizes_f) == 231
    assert f["T1"].shape == (997, 3)
    assert all(f[k].shape[1] == 2 for k in f.files if k != "T1")


@pytest.mark.parametrize("key", ["S1", "F9", "T1"])
def test_noiseless_problem_maps_back_exactly(key):
    model = _models()[key]
    D = model.shape[1]
    P = synth.simulation(model, 3, rand_noise=0.0, rand_outliers=0, rand_miss_rate=0.0)
    assert np.allclose(P.R_G @ P.R_G.T, np.eye(D), atol=1e-14) and np.linalg.det(P.R_G) > 0
    back = P.Y @ P.R_G.T + P.t_G
    d2 = ((back[:, None, :] - model[None, :, :]) ** 2).sum(-1).min(axis=1)
    assert d2.max() < 1e-28
    d2x = ((P.X[:, None, :] - model[None, :, :]) ** 2).sum(-1).min(axis=1)
    assert d2x.max() == 0.0
    # the sampling rates of noise_and_sampling2D/3D.m: 0.9 of the points for X, 0.85 for Y
    assert 0.8 * len(model) < P.N <= len(model) and 0.75 * len(model) < P.M <= len(model)


@pytest.mark.parametrize("key", ["F7", "T1"])
def test_covariances_and_ranges(key):
    model = _models()[key]
    D = model.shape[1]
    out_max = 50 if D == 2 else 100
    for trial in range(5):
        P = synth.simulation(model, trial)
        off = ~np.eye(D, dtype=bool)
        assert np.all(P.X_C[:, off] == 0) and np.all(np.diagonal(P.X_C, axis1=1, axis2=2) >= 1.0)   # exp(3.4657 |r|)
        back = P.R_G @ P.Y_C @ P.R_G.T                      # Y's covariances, rotated back
        assert np.allclose(back[:, off], 0, atol=1e-12) and np.all(np.diagonal(back, axis1=1, axis2=2) >= 1.0 - 1e-12)
        assert _deg(P.R_G) <= (30 if D == 2 else 30 * math.sqrt(3)) + 1e-9
        assert np.all(np.abs(P.R_G.T @ -P.t_G) <= 0.5 + 1e-12)
        assert P.N <= len(model) + out_max and P.M <= len(model) + out_max
    a, b = synth.simulation(model, 2), synth.simulation(model, 2)
    assert np.array_equal(a.X, b.X) and np.array_equal(a.Y_C, b.Y_C)


@pytest.mark.gpu
@pytest.mark.parametrize("models", ["S", "F", "T"])
def test_registration_on_the_simulation_protocol(models):
    from dugma_b200 import evaluate
    rows = [evaluate.register(P, 0, 700) for P, _ in evaluate.scenes_simulation(FIX, models, 20)]
    deg = np.array([r["deg"] for r in rows])
    print(models, "median deg", np.median(deg), "within 2 deg", np.mean(deg < 2), "worst", deg.max())
    assert np.median(deg) < 1.0
    assert np.mean(deg < 2.0) >= 0.85
