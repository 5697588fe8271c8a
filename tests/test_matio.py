"""MATLAB layout conversion, .mat round trips, and the reference's own data files (CPU)."""
import os

import numpy as np
import pytest

from dugma_b200 import matio, synth


@pytest.mark.parametrize("D", [3, 2])
def test_block_layout_matches_reference_convention(D):
    # covariance of point k is X_C(:, D(k-1)+1 : Dk) (1-based MATLAB columns)
    n = 5
    C = np.arange(n * D * D, dtype=float).reshape(n, D, D) + 0.5
    M = matio.cov_to_matlab(C)
    assert M.shape == (D, D * n)
    for k in range(n):
        assert np.array_equal(M[:, D * k:D * (k + 1)], C[k])
    assert np.array_equal(matio.cov_from_matlab(M, D), C)
    # column-major storage of the D x (D n) matrix is the C ABI's per-point block layout
    flat = M.reshape(-1, order="F")
    assert np.array_equal(flat, np.transpose(C, (0, 2, 1)).reshape(-1))


def test_cloud_layout():
    X = np.arange(12, dtype=float).reshape(4, 3)
    A = matio.cloud_to_matlab(X)
    assert A.shape == (3, 4) and np.array_equal(A[:, 2], X[2])
    assert np.array_equal(A.reshape(-1, order="F"), X.reshape(-1))
    assert np.array_equal(matio.cloud_from_matlab(A), X)


def test_mat_round_trip(tmp_path):
    P = synth.workload0(n=64)
    path = str(tmp_path / "p.mat")
    matio.save_problem(path, P)
    Q = matio.load_problem(path)
    for a in ("X", "Y", "X_C", "Y_C", "R_G", "t_G"):
        assert np.array_equal(getattr(P, a), getattr(Q, a)), a


def test_mat_errors(tmp_path):
    from scipy.io import savemat
    path = str(tmp_path / "bad.mat")
    savemat(path, {"X": np.zeros((3, 4)), "Y": np.zeros((3, 5)), "X_C": np.zeros((3, 12)),
                   "Y_C": np.zeros((3, 14))})
    with pytest.raises(ValueError):
        matio.load_problem(path)
    savemat(path, {"X": np.zeros((3, 4))})
    with pytest.raises(KeyError):
        matio.load_problem(path)


def test_load_single_precision_model_cloud(tmp_path):
    from scipy.io import savemat
    X = np.random.default_rng(0).standard_normal((3, 17)).astype(np.float32)
    path = str(tmp_path / "model.mat")
    savemat(path, {"X": X})
    got = matio.load_cloud(path)
    assert got.shape == (17, 3) and got.dtype == np.float64
    assert np.array_equal(got, X.T.astype(np.float64))


def _ref_file(*parts):
    from oracle.ref_build import reference_tree
    ref = reference_tree()
    if ref is None:
        pytest.skip("reference tree not present (DUGMA_REFERENCE)")
    return os.path.join(ref, *parts)


def test_reads_a_reference_kinect_scene():
    """dataset_all/Kinect_Application/1.mat through load_problem: 3 x N clouds, 3 x 3N covariance
    blocks (the covariance of X(:, k) is X_C(:, 3(k-1)+1 : 3k), dataset_all "Read Me"), ground truth."""
    from scipy.io import loadmat
    path = _ref_file("dataset_all", "Kinect_Application", "1.mat")
    P = matio.load_problem(path)
    m = loadmat(path)
    assert P.X.shape == (m["X"].shape[1], 3) and P.Y.shape == (m["Y"].shape[1], 3)
    assert P.X_C.shape == (P.N, 3, 3) and P.Y_C.shape == (P.M, 3, 3)
    for k in (0, 1, P.N - 1):
        assert np.array_equal(P.X[k], m["X"][:, k])
        assert np.array_equal(P.X_C[k], m["X_C"][:, 3 * k:3 * k + 3])
    assert np.array_equal(P.Y_C[7], m["Y_C"][:, 21:24])
    assert np.allclose(P.R_G @ P.R_G.T, np.eye(3), atol=1e-6) and P.t_G.shape == (3,)
    # the fixture made from it holds the same scene
    f = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "kinect_scenes.npz"))
    assert np.allclose(f["X1"], P.X, rtol=1e-7, atol=0)
    assert np.array_equal(f["cx1"].astype(float), P.X_C[:, 0, 0])
    assert np.array_equal(f["RG1"], P.R_G)


def test_reads_a_reference_2d_shape_model():
    path = _ref_file("dataset_all", "2D_SHAPE_MODEL", "1.mat")
    X = matio.load_cloud(path)
    assert X.shape[1] == 2 and X.shape[0] > 10 and np.all(np.isfinite(X))
