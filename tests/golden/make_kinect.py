"""Fixture of the reference's 30 real Kinect scenes and the authors' recorded poses (test data).

    python tests/golden/make_kinect.py [REFERENCE_TREE]

Reads, from the reference tree (DUGMA_REFERENCE or the recipe default of
oracle/ref_build.py):
  dataset_all/Kinect_Application/{k}.mat            X, Y (3 x N), X_C, Y_C (3 x 3N), R_G, t_G
  Our_result_in_Kinect_Application/Ours_{k}_result.mat   R, t (the authors' registration),
                                                          time_stop_DUGMA (their seconds)
for k = 1..30 (the layout of dataset_all "Read Me") and writes tests/golden/kinect_scenes.npz:
  X{k}, Y{k}     (N, 3) float32 coordinates (the library's device state is FP32; rounding the
                 stored doubles moves a point by < 1e-7 relative)
  cx{k}, cy{k}   (N,) float32: every covariance block of these scenes is c I, so c is stored
                 (NaN where the dataset's block is NaN: the reference's init neglects those
                 points, init.cu:86-100, as the library does)
  RG{k}, tG{k}   ground truth;  Ra{k}, ta{k}, sa{k}  the authors' pose and seconds.
The script checks the isotropy it relies on and fails otherwise.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "kinect_scenes.npz")


def _iso_scalar(C: np.ndarray) -> np.ndarray:
    """3 x 3N covariance blocks that are all c I (or all NaN) -> c per point."""
    b = C.reshape(3, -1, 3).transpose(1, 0, 2)
    c = b[:, 0, 0].copy()
    nan = np.isnan(b).any(axis=(1, 2))
    iso = np.einsum("n,ab->nab", c, np.eye(3))
    if not np.array_equal(b[~nan], iso[~nan]):
        raise ValueError("a covariance block is not a multiple of the identity")
    c[nan] = np.nan
    if not np.array_equal(c[~nan].astype(np.float32).astype(np.float64), c[~nan]):
        raise ValueError("a covariance scale is not exact in float32")
    return c.astype(np.float32)


def main(ref: str) -> None:
    from scipy.io import loadmat
    out = {}
    for k in range(1, 31):
        d = loadmat(os.path.join(ref, "dataset_all", "Kinect_Application", f"{k}.mat"))
        r = loadmat(os.path.join(ref, "Our_result_in_Kinect_Application", f"Ours_{k}_result.mat"))
        out[f"X{k}"] = np.ascontiguousarray(d["X"].T, dtype=np.float32)
        out[f"Y{k}"] = np.ascontiguousarray(d["Y"].T, dtype=np.float32)
        out[f"cx{k}"] = _iso_scalar(d["X_C"])
        out[f"cy{k}"] = _iso_scalar(d["Y_C"])
        out[f"RG{k}"] = np.asarray(d["R_G"], dtype=np.float64)
        out[f"tG{k}"] = np.asarray(d["t_G"], dtype=np.float64).reshape(3)
        out[f"Ra{k}"] = np.asarray(r["R"], dtype=np.float64)
        out[f"ta{k}"] = np.asarray(r["t"], dtype=np.float64).reshape(3)
        out[f"sa{k}"] = np.float64(np.asarray(r["time_stop_DUGMA"]).reshape(-1)[0])
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT} ({os.path.getsize(OUT) / 1e6:.2f} MB)")


if __name__ == "__main__":
    sys.path.insert(0, ROOT)
    from oracle.ref_build import reference_tree
    ref = sys.argv[1] if len(sys.argv) > 1 else reference_tree()
    if not ref:
        raise SystemExit("the reference tree is not present (pass it or set DUGMA_REFERENCE)")
    main(ref)
