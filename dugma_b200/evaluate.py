"""Registration accuracy and time over two-view scenes.

    python -m dugma_b200.evaluate [--mode 0|1] [--max-iteration 300]
                                  [--scenes 30 | --mat-dir DIR [--results-dir DIR] | --npz FILE |
                                   --sim FILE [--models S|F|T] [--trials 100]]

Scenes come from the seeded synthetic stand-ins (synth.kinect_like, default), from a
directory of .mat files in the reference dataset's layout ({k}.mat holding X, Y, X_C, Y_C,
R_G, t_G; dataset_all "Read Me"), optionally with a directory of recorded results
(Ours_{k}_result.mat holding R, t) to compare against, or from an .npz holding the same
scenes (X{k}, Y{k} point rows, cx{k}, cy{k} isotropic covariance scales, RG{k}, tG{k} and the
recorded Ra{k}, ta{k}, sa{k}), or drawn by the reference's simulation protocol from its 2D model
contours and 3D model surface in tests/golden/sim_models.npz (--sim; main_simulation.m:17-35,
whose settings differ only in allowing 700 iterations, line 47).  Each scene is registered from the identity pose with the
settings of main_kinect_real_application.m:14-17 (300 iterations, rotation / translation /
sigma tolerances 1e-4 / 1e-8 / 1e-9) and scored with its error measures (lines 33-35 there):
||I - R pinv(R_G)||_F and ||t - t_G||, plus the geodesic rotation angle, and, where a
recorded result exists, the angle between R and the recorded rotation and ||t - t_recorded||.
Mode 0 is the reference's loop (surrogate coefficients + constrained minimisation per sigma
step), mode 1 the direct quasi-Newton on the fused adjoint.  One JSON line per scene, then a
summary line with medians.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import re
import time

import numpy as np

from . import api, synth
from .pose import rotation_error_deg
from .synth import Problem


def _angle_deg(R, R_G) -> float:
    """The rotation angle between R and R_G in degrees (2D or 3D)."""
    if np.asarray(R).shape[0] == 2:
        Q = np.asarray(R) @ np.asarray(R_G).T
        return abs(math.degrees(math.atan2(Q[1, 0], Q[0, 0])))
    return rotation_error_deg(R, R_G)


def register(P: Problem, mode: int = 0, max_iteration: int = 300, recorded=None) -> dict:
    """Register one scene from the identity pose; recorded = (R, t[, seconds]) or None."""
    D = P.X.shape[1]
    t0 = time.perf_counter()
    R, t, stats = api.DUGMA(P.X, P.Y, P.X_C, P.Y_C, np.eye(D), np.zeros(D), Max_Iteration=max_iteration,
                            accuracy_rotation=1e-4, accuracy_translation=1e-8, accuracy_sig=1e-9, mode=mode)
    wall = time.perf_counter() - t0
    row = {"scene": P.name, "N": P.N, "M": P.M,
           "error_R": float(np.linalg.norm(np.eye(D) - R @ np.linalg.pinv(P.R_G))),
           "error_t": float(np.linalg.norm(t - P.t_G)),
           "deg": _angle_deg(R, P.R_G), "iterations": int(stats[0]), "seconds": wall}
    if recorded is not None:
        Ra, ta = recorded[0], recorded[1]
        row["recorded_error_R"] = float(np.linalg.norm(np.eye(3) - Ra @ np.linalg.pinv(P.R_G)))
        row["recorded_error_t"] = float(np.linalg.norm(ta - P.t_G))
        row["vs_recorded_deg"] = _angle_deg(R, Ra)
        row["vs_recorded_t"] = float(np.linalg.norm(t - ta))
        if len(recorded) > 2:
            row["recorded_seconds"] = float(recorded[2])
    return row


def scenes_synthetic(n: int):
    for k in range(n):
        yield synth.kinect_like(k), None


def _numbered(dir_: str, pattern: str):
    rx = re.compile(pattern)
    found = []
    for f in os.listdir(dir_):
        m = rx.fullmatch(f)
        if m:
            found.append((int(m.group(1)), os.path.join(dir_, f)))
    return sorted(found)


def scenes_from_mat(mat_dir: str, results_dir: str | None = None):
    """{k}.mat scenes in numeric order, with Ours_{k}_result.mat from results_dir if given."""
    from scipy.io import loadmat
    from .matio import load_problem
    for k, path in _numbered(mat_dir, r"(\d+)\.mat"):
        P = load_problem(path)
        rec = None
        if results_dir:
            rp = os.path.join(results_dir, f"Ours_{k}_result.mat")
            if os.path.exists(rp):
                r = loadmat(rp)
                rec = (np.asarray(r["R"], float), np.asarray(r["t"], float).reshape(-1))
        yield P, rec


def scenes_from_npz(path: str):
    """Scenes of an .npz in the layout of the module docstring, in numeric order."""
    f = np.load(path)
    ks = sorted(int(m.group(1)) for m in (re.fullmatch(r"X(\d+)", n) for n in f.files) if m)
    for k in ks:
        X, Y = f[f"X{k}"].astype(np.float64), f[f"Y{k}"].astype(np.float64)
        D = X.shape[1]
        XC = np.einsum("n,ab->nab", f[f"cx{k}"].astype(np.float64), np.eye(D))
        YC = np.einsum("n,ab->nab", f[f"cy{k}"].astype(np.float64), np.eye(D))
        P = Problem(X, Y, XC, YC, f[f"RG{k}"], f[f"tG{k}"], f"scene{k}")
        rec = None
        if f"Ra{k}" in f.files:
            rec = (f[f"Ra{k}"], f[f"ta{k}"], float(f[f"sa{k}"])) if f"sa{k}" in f.files else (f[f"Ra{k}"], f[f"ta{k}"])
        yield P, rec


def scenes_simulation(path: str, models: str = "S", trials: int = 100):
    """The reference's simulation (main_simulation.m:17-56, produce_point_cloud.m) on the models
    of an .npz written by tests/golden/make_sim_models.py: trial k draws a problem from model
    (k mod 100) + 1 of the set with the generator restated in synth.simulation.  models: "S"
    (2D_SHAPE_MODEL), "F" (2D_Fish_MODEL, 200 points) or "T" (the 3D_SHAPE surface, the one
    3D model released)."""
    f = np.load(path)
    for k in range(trials):
        key = "T1" if models == "T" else f"{models}{k % 100 + 1}"
        yield synth.simulation(f[key], k, name=f"{key}_trial{k}"), None


def summarise(rows, mode) -> dict:
    summ = {"scenes": len(rows), "mode": mode}
    for key in ("error_R", "error_t", "deg", "iterations", "seconds", "vs_recorded_deg", "vs_recorded_t",
                "recorded_error_R", "recorded_error_t", "recorded_seconds"):
        v = np.array([r[key] for r in rows if key in r], dtype=float)
        if v.size:
            summ[key] = {"median": float(np.median(v)), "mean": float(v.mean()), "max": float(v.max())}
    return summ


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--scenes", type=int, default=30, help="synthetic stand-in scenes")
    ap.add_argument("--mat-dir", default="", help="directory of {k}.mat scenes in the reference layout")
    ap.add_argument("--results-dir", default="", help="directory of Ours_{k}_result.mat recorded results")
    ap.add_argument("--npz", default="", help=".npz of scenes (see the module docstring)")
    ap.add_argument("--sim", default="", help=".npz of simulation models (tests/golden/sim_models.npz): the "
                                             "reference's simulation protocol")
    ap.add_argument("--models", default="S", help="with --sim: S (2D shapes), F (2D fish) or T (3D)")
    ap.add_argument("--trials", type=int, default=100, help="with --sim: problems drawn")
    ap.add_argument("--mode", type=int, default=0)
    ap.add_argument("--max-iteration", type=int, default=0, help="default 300, or 700 with --sim "
                                                                  "(main_simulation.m:47)")
    a = ap.parse_args(argv)
    if a.sim:
        src = scenes_simulation(a.sim, a.models, a.trials)
    elif a.npz:
        src = scenes_from_npz(a.npz)
    elif a.mat_dir:
        src = scenes_from_mat(a.mat_dir, a.results_dir or None)
    else:
        src = scenes_synthetic(a.scenes)
    max_it = a.max_iteration or (700 if a.sim else 300)
    rows = []
    for P, rec in src:
        r = register(P, a.mode, max_it, rec)
        rows.append(r)
        print(json.dumps(r), flush=True)
    print(json.dumps({"summary": summarise(rows, a.mode)}), flush=True)


if __name__ == "__main__":
    main()
