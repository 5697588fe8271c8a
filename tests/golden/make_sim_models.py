"""Fixture of the model contours and surface of the reference's simulation (test data).

    python tests/golden/make_sim_models.py [REFERENCE_TREE]

Reads, from the reference tree (DUGMA_REFERENCE or the recipe default of
oracle/ref_build.py):
  dataset_all/2D_SHAPE_MODEL/{k}.mat                  X (2 x N): 100 shape contours, N 206..532
  dataset_all/2D_Fish_MODEL/dataset2D_200/{k}.mat     X (2 x N): 100 fish contours, N 162..231
  dataset_all/3D_SHAPE/1.mat                          X (3 x N): the one released 3D model, N 997
(the models main_simulation.m:23-35 loads through produce_point_cloud.m:23-27) and writes
tests/golden/sim_models.npz with S{k}, F{k} (k = 1..100) and T1, the (N, D) float64 model
points.  The registration problems are drawn from them by the seeded generator restated in
dugma_b200/synth.py (simulation).
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "sim_models.npz")


def _model(path: str, D: int) -> np.ndarray:
    from scipy.io import loadmat
    X = np.asarray(loadmat(path)["X"], dtype=np.float64)
    if X.ndim != 2 or X.shape[0] != D:
        raise ValueError(f"{path}: X is {X.shape}, expected {D} x N")
    return np.ascontiguousarray(X.T)


def main(ref: str) -> None:
    ds = os.path.join(ref, "dataset_all")
    out = {}
    for k in range(1, 101):
        out[f"S{k}"] = _model(os.path.join(ds, "2D_SHAPE_MODEL", f"{k}.mat"), 2)
        out[f"F{k}"] = _model(os.path.join(ds, "2D_Fish_MODEL", "dataset2D_200", f"{k}.mat"), 2)
    out["T1"] = _model(os.path.join(ds, "3D_SHAPE", "1.mat"), 3)
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT} ({os.path.getsize(OUT) / 1e6:.2f} MB)")


if __name__ == "__main__":
    sys.path.insert(0, ROOT)
    from oracle.ref_build import reference_tree
    ref = sys.argv[1] if len(sys.argv) > 1 else reference_tree()
    if not ref:
        raise SystemExit("the reference tree is not present (pass it or set DUGMA_REFERENCE)")
    main(ref)
