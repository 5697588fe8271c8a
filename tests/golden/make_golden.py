"""Record the reference plugins' outputs as golden fixtures (run on a GPU).

    python tests/golden/make_golden.py [out_dir [case ...]]

Runs the reference's own init / update_sig / compi (built from its sources by
oracle/ref_build.py into oracle/_ref) on small seeded inputs (well and ill conditioned, equal
and uneven sizes, 3D and 2D, with and without non-positive-definite covariances) -- and on 2048
points of each view of the reference's own Kinect scene 1 -- and stores inputs and outputs in
tests/golden/ref_<case>.npz:
  inputs   X, X_C, Y, Y_C (float64), poses R (k, D, D), t (k, D)
  outputs  the FP32 device state after init (d_X, inverse covariances, d_Y, ..., det_X,
           det_Y), sig from update_sig at each pose, the 640 compi coefficients at each
           pose (with that pose's sig).
Sizes are multiples of 32: the reference compi kernel is only well defined there.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from dugma_b200 import synth  # noqa: E402
from dugma_b200.pose import expmap, rot2d  # noqa: E402
from oracle import ref_plugins  # noqa: E402


def _dev_f32(ptr, n):
    import torch

    class A:
        def __init__(self):
            self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f4", "data": (ptr, False), "version": 3}

    return torch.as_tensor(A(), device="cuda").cpu().numpy().copy()


def cases():
    rng = np.random.default_rng(2024)
    # 1: the 1K sphere workload at 512 points
    P = synth.workload0(n=512)
    yield "sphere512", P.X, P.X_C, P.Y, P.Y_C, [np.eye(3), P.R_G @ expmap([0.05, -0.08, 0.1])], \
        [np.zeros(3), P.t_G + 0.01]
    # 2: random covariances with non-positive-definite points
    n, m = 64, 96
    X = rng.standard_normal((n, 3)) * 0.5
    Y = X[np.arange(m) % n] @ expmap([0.2, 0.1, -0.3]).T + 0.1 + 0.03 * rng.standard_normal((m, 3))
    A = rng.standard_normal((n, 3, 3)) * 0.2
    XC = A @ np.transpose(A, (0, 2, 1)) + 0.02 * np.eye(3)
    B = rng.standard_normal((m, 3, 3)) * 0.2
    YC = B @ np.transpose(B, (0, 2, 1)) + 0.02 * np.eye(3)
    XC[5] = np.diag([-1.0, 1.0, 1.0])
    YC[7] = np.diag([1.0, 1.0, -3.0])
    yield "random64x96", X, XC, Y, YC, [expmap([0.1, 0.2, -0.1]), np.eye(3)], [np.array([0.05, -0.1, 0.0]), np.zeros(3)]
    # 3: 2D
    n, m = 320, 256
    th = rng.uniform(0, 2 * np.pi, n)
    X = np.stack([np.cos(th) * (1 + 0.2 * np.sin(5 * th)), np.sin(th) * (1 + 0.2 * np.sin(5 * th))], 1)
    th2 = rng.uniform(0, 2 * np.pi, m)
    S = np.stack([np.cos(th2) * (1 + 0.2 * np.sin(5 * th2)), np.sin(th2) * (1 + 0.2 * np.sin(5 * th2))], 1)
    Y = S @ rot2d(0.5).T + np.array([0.1, -0.2]) + 0.01 * rng.standard_normal((m, 2))
    XC = np.einsum("n,ab->nab", rng.uniform(1e-3, 4e-3, n), np.eye(2)) + np.einsum(
        "n,ab->nab", rng.uniform(0, 1e-3, n), np.array([[0, 1.0], [1.0, 0]]))
    YC = np.einsum("n,ab->nab", rng.uniform(1e-3, 4e-3, m), np.eye(2))
    yield "curve2d_320x256", X, XC, Y, YC, [np.eye(2), rot2d(-0.4)], [np.zeros(2), np.array([-0.1, 0.2])]
    # 4: real data -- Kinect scene 1 of the reference's dataset (tests/golden/kinect_scenes.npz), 2048
    # points of each view drawn without replacement, normalised as DUGMA.m:19-32 does before its
    # init call (covariances unscaled), at the identity and at the authors' recorded pose
    f = np.load(os.path.join(ROOT, "tests", "golden", "kinect_scenes.npz"))
    X0, Y0 = f["X1"].astype(np.float64), f["Y1"].astype(np.float64)
    cx, cy = f["cx1"].astype(np.float64), f["cy1"].astype(np.float64)
    ix = np.sort(rng.choice(len(X0), 2048, replace=False))
    iy = np.sort(rng.choice(len(Y0), 2048, replace=False))
    X, Y = X0[ix], Y0[iy]
    XC, YC = np.einsum("n,ab->nab", cx[ix], np.eye(3)), np.einsum("n,ab->nab", cy[iy], np.eye(3))
    xd, yd = X.mean(axis=0), Y.mean(axis=0)
    scale = max(np.sqrt(((X - xd) ** 2).sum(1).mean()), np.sqrt(((Y - yd) ** 2).sum(1).mean()))
    X, Y = (X - xd) / scale, (Y - yd) / scale
    Ra, ta = f["Ra1"], f["ta1"]
    yield "kinect1_2048", X, XC, Y, YC, [np.eye(3), Ra], [np.zeros(3), (ta - xd + Ra @ yd) / scale]
    # 5: the ill-conditioned sphere (10 % outliers, 8-NN sample covariances with eigenvalues
    # clamped to [1e-6, 1e-2], condition up to ~7e3) at 2048 points, near the ground truth and at it
    P = synth.workload1(n=2048)
    yield "illcond2048", P.X, P.X_C, P.Y, P.Y_C, [P.R_G @ expmap([0.02, -0.03, 0.01]), P.R_G], \
        [P.t_G + 0.005, P.t_G]
    # 6: clouds of different sizes -- 1024 sources against 3072 targets of the harmonic surface
    P = synth.workload2(n=3072)
    yield "uneven1024x3072", P.X[:1024], P.X_C[:1024], P.Y, P.Y_C, [np.eye(3), P.R_G @ expmap([0.05, 0.0, -0.04])], \
        [np.zeros(3), P.t_G - 0.01]
    # 7: 2D, uneven sizes, with covariances that are not positive definite on both sides
    n, m = 224, 416
    th = rng.uniform(0, 2 * np.pi, n)
    X = np.stack([1.2 * np.cos(th), 0.8 * np.sin(th) * (1 + 0.3 * np.cos(3 * th))], 1)
    th2 = rng.uniform(0, 2 * np.pi, m)
    S = np.stack([1.2 * np.cos(th2), 0.8 * np.sin(th2) * (1 + 0.3 * np.cos(3 * th2))], 1)
    Y = S @ rot2d(-0.3).T + np.array([-0.05, 0.15]) + 0.01 * rng.standard_normal((m, 2))
    A = rng.standard_normal((n, 2, 2)) * 0.05
    XC = A @ np.transpose(A, (0, 2, 1)) + 1e-3 * np.eye(2)
    B = rng.standard_normal((m, 2, 2)) * 0.05
    YC = B @ np.transpose(B, (0, 2, 1)) + 1e-3 * np.eye(2)
    XC[3] = np.diag([-1e-3, 2e-3])
    XC[100] = np.array([[1e-3, 2e-3], [2e-3, 1e-3]])
    YC[11] = np.diag([2e-3, 0.0])
    yield "curve2d_nonpd_224x416", X, XC, Y, YC, [np.eye(2), rot2d(0.25)], [np.zeros(2), np.array([0.05, -0.1])]


def main(out_dir, only=None):
    os.makedirs(out_dir, exist_ok=True)
    for name, X, XC, Y, YC, Rs, ts in cases():
        if only and name not in only:
            continue
        N, D = X.shape
        M = Y.shape[0]
        ptr = ref_plugins.init(X, XC, Y, YC)
        p = [ptr[k] for k in range(6)]
        state = {"d_X": _dev_f32(p[0], N * D), "d_X_C": _dev_f32(p[1], N * D * D), "d_Y": _dev_f32(p[2], M * D),
                 "d_Y_C": _dev_f32(p[3], M * D * D), "det_X": _dev_f32(p[4], N), "det_Y": _dev_f32(p[5], M)}
        sigs, coefs = [], []
        for R, t in zip(Rs, ts):
            s = ref_plugins.update_sig(ptr, R, t, N, M, D)
            sigs.append(s)
            coefs.append(ref_plugins.compi(ptr, R, t, N, M, D, s))
        np.savez_compressed(os.path.join(out_dir, f"ref_{name}.npz"), X=X, X_C=XC, Y=Y, Y_C=YC, R=np.array(Rs),
                            t=np.array(ts), sig=np.array(sigs, np.float32), coef=np.array(coefs), **state)
        print(name, "sig", sigs, "coef[0:3]", [c[:3] for c in coefs])


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(ROOT, "tests", "golden"), sys.argv[2:] or None)
