"""MATLAB data layout and .mat ingest for the registration entry points.

The reference passes clouds as D x N matrices (one point per column, DUGMA.m:19) and
covariances as D x (D N) matrices whose columns D(k-1)+1 .. Dk hold the covariance of
point k (dataset_all "Read Me":7-8).  In MATLAB's column-major storage both are already
the point-major C arrays the C ABI takes (X[k*D + a], X_C[k*D*D + a + D*b]); this module
converts between them and numpy's (N, D) / (N, D, D) views, and reads or writes .mat
files (MATLAB v5-v7.2 through scipy.io) holding X, Y, X_C, Y_C and optionally the ground
truth R_G, t_G.
"""
from __future__ import annotations

import numpy as np

from .synth import Problem


def cloud_from_matlab(A) -> np.ndarray:
    """D x N MATLAB cloud -> (N, D) float64."""
    A = np.asarray(A, dtype=np.float64)
    if A.ndim != 2 or A.shape[0] not in (2, 3):
        raise ValueError(f"a cloud is D x N with D in {{2, 3}}, got {A.shape}")
    return np.ascontiguousarray(A.T)


def cloud_to_matlab(X) -> np.ndarray:
    """(N, D) -> D x N."""
    return np.asarray(X, dtype=np.float64).T.copy()


def cov_from_matlab(C, D: int) -> np.ndarray:
    """D x (D N) MATLAB covariance blocks -> (N, D, D), block k = C(:, D(k-1)+1 : Dk)."""
    C = np.asarray(C, dtype=np.float64)
    if C.ndim != 2 or C.shape[0] != D or C.shape[1] % D:
        raise ValueError(f"covariances are {D} x ({D} N), got {C.shape}")
    n = C.shape[1] // D
    return np.ascontiguousarray(C.reshape(D, n, D).transpose(1, 0, 2))


def cov_to_matlab(C) -> np.ndarray:
    """(N, D, D) -> D x (D N)."""
    C = np.asarray(C, dtype=np.float64)
    n, D, _ = C.shape
    return C.transpose(1, 0, 2).reshape(D, n * D).copy()


def load_cloud(path: str, var: str = "X") -> np.ndarray:
    """Read one D x N cloud (single or double) from a .mat file -> (N, D) float64 (the
    dataset's shape-model files hold a single model cloud X)."""
    from scipy.io import loadmat
    m = loadmat(path)
    if var not in m:
        raise KeyError(f"{path}: no variable {var!r}")
    return cloud_from_matlab(m[var])


def load_problem(path: str, x: str = "X", y: str = "Y", x_cov: str = "X_C", y_cov: str = "Y_C",
                 r_gt: str = "R_G", t_gt: str = "t_G") -> Problem:
    """Read a registration problem from a .mat file in the reference's layout.  The ground
    truth is optional (identity / zero when the file has none)."""
    from scipy.io import loadmat
    m = loadmat(path)
    for key in (x, y, x_cov, y_cov):
        if key not in m:
            raise KeyError(f"{path}: no variable {key!r}")
    X, Y = cloud_from_matlab(m[x]), cloud_from_matlab(m[y])
    D = X.shape[1]
    if Y.shape[1] != D:
        raise ValueError(f"{path}: X is {D}-D but Y is {Y.shape[1]}-D")
    XC, YC = cov_from_matlab(m[x_cov], D), cov_from_matlab(m[y_cov], D)
    if XC.shape[0] != X.shape[0] or YC.shape[0] != Y.shape[0]:
        raise ValueError(f"{path}: covariance count differs from point count")
    R = np.asarray(m[r_gt], dtype=np.float64) if r_gt in m else np.eye(D)
    t = np.asarray(m[t_gt], dtype=np.float64).reshape(-1) if t_gt in m else np.zeros(D)
    name = path.rsplit("/", 1)[-1]
    return Problem(X, Y, XC, YC, R, t, name)


def save_problem(path: str, P: Problem) -> None:
    """Write a problem in the reference's layout (X, Y, X_C, Y_C, R_G, t_G)."""
    from scipy.io import savemat
    savemat(path, {"X": cloud_to_matlab(P.X), "Y": cloud_to_matlab(P.Y), "X_C": cov_to_matlab(P.X_C),
                   "Y_C": cov_to_matlab(P.Y_C), "R_G": np.asarray(P.R_G, dtype=np.float64),
                   "t_G": np.asarray(P.t_G, dtype=np.float64).reshape(-1, 1)})
