"""MATLAB layout conversion and .mat round trips (CPU)."""
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
