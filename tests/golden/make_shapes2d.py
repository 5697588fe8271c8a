"""Fixture of the reference's 2D model contours (test data for the 2D simulation protocol).

    python tests/golden/make_shapes2d.py [REFERENCE_TREE]

Reads, from the reference tree (DUGMA_REFERENCE or the recipe default of
oracle/ref_build.py):
  dataset_all/2D_SHAPE_MODEL/{k}.mat                  X (2 x N): 100 shape contours, N 206..532
  dataset_all/2D_Fish_MODEL/dataset2D_200/{k}.mat     X (2 x N): 100 fish contours, N 162..231
for k = 1..100 (the models main_simulation.m:23-28 loads through produce_point_cloud.m:23-27)
and writes tests/golden/shapes2d.npz with S{k} and F{k}, the (N, 2) float64 model points.
The registration problems are drawn from them by the seeded generator restated in
dugma_b200/synth.py (simulation2d).
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "shapes2d.npz")


def main(ref: str) -> None:
    from scipy.io import loadmat
    out = {}
    for prefix, sub in (("S", ("2D_SHAPE_MODEL",)), ("F", ("2D_Fish_MODEL", "dataset2D_200"))):
        for k in range(1, 101):
            X = np.asarray(loadmat(os.path.join(ref, "dataset_all", *sub, f"{k}.mat"))["X"], dtype=np.float64)
            if X.ndim != 2 or X.shape[0] != 2:
                raise ValueError(f"{sub} {k}.mat: X is {X.shape}, expected 2 x N")
            out[f"{prefix}{k}"] = np.ascontiguousarray(X.T)
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT} ({os.path.getsize(OUT) / 1e6:.2f} MB)")


if __name__ == "__main__":
    sys.path.insert(0, ROOT)
    from oracle.ref_build import reference_tree
    ref = sys.argv[1] if len(sys.argv) > 1 else reference_tree()
    if not ref:
        raise SystemExit("the reference tree is not present (pass it or set DUGMA_REFERENCE)")
    main(ref)
