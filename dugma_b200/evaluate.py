"""Registration accuracy and time over seeded two-view depth scenes.

    python -m dugma_b200.evaluate [--scenes 30] [--mode 0|1] [--max-iteration 300]

Each scene (synth.kinect_like) is registered from the identity pose with the settings of
main_kinect_real_application.m:14-17 (300 iterations, rotation / translation / sigma
tolerances 1e-4 / 1e-8 / 1e-9), and scored with its error measures (lines 33-35 there):
||I - R pinv(R_G)||_F and ||t - t_G||, plus the geodesic rotation angle.  Mode 0 is the
reference's loop (surrogate coefficients + constrained minimisation per sigma step),
mode 1 the direct quasi-Newton on the fused adjoint.  One JSON line per scene, then a
summary line with medians.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import api, synth
from .pose import rotation_error_deg


def register_scene(k: int, mode: int = 0, max_iteration: int = 300) -> dict:
    P = synth.kinect_like(k)
    t0 = time.perf_counter()
    R, t, stats = api.DUGMA(P.X, P.Y, P.X_C, P.Y_C, np.eye(3), np.zeros(3), Max_Iteration=max_iteration,
                            accuracy_rotation=1e-4, accuracy_translation=1e-8, accuracy_sig=1e-9, mode=mode)
    wall = time.perf_counter() - t0
    return {"scene": P.name, "N": P.N, "M": P.M,
            "error_R": float(np.linalg.norm(np.eye(3) - R @ np.linalg.pinv(P.R_G))),
            "error_t": float(np.linalg.norm(t - P.t_G)),
            "deg": rotation_error_deg(R, P.R_G), "iterations": int(stats[0]), "seconds": wall}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--scenes", type=int, default=30)
    ap.add_argument("--mode", type=int, default=0)
    ap.add_argument("--max-iteration", type=int, default=300)
    a = ap.parse_args(argv)
    rows = []
    for k in range(a.scenes):
        r = register_scene(k, a.mode, a.max_iteration)
        rows.append(r)
        print(json.dumps(r), flush=True)
    summ = {"scenes": len(rows), "mode": a.mode}
    for key in ("error_R", "error_t", "deg", "iterations", "seconds"):
        v = np.array([r[key] for r in rows], dtype=float)
        summ[key] = {"median": float(np.median(v)), "mean": float(v.mean()), "max": float(v.max())}
    print(json.dumps({"summary": summ}), flush=True)


if __name__ == "__main__":
    main()
