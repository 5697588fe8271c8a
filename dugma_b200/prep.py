"""Host-side scale helpers of the reference's MATLAB code, for callers porting its scripts.

    normalize(X, Y)  -> (Xn, Yn, Normal)    normalize.m:3-26 (the registration driver applies
                                             the same in C++ before it uploads the clouds)
    get_sd(X, Y)     -> Scales              get_sd2D.m / get_sd3D.m
    get_radius(X)    -> Radius              get_radius.m

Clouds are (N, D) arrays (one point per row).  Each cloud is centred on its own mean; the
scale is the RMS distance to that mean, sqrt(sum |x - mean|^2 / N); normalize divides both
clouds by the larger of the two scales.  Covariances are not rescaled (DUGMA.m passes them
unchanged).
"""
from __future__ import annotations

import dataclasses

import numpy as np


@dataclasses.dataclass
class Normal:
    xd: np.ndarray      # mean of X
    yd: np.ndarray      # mean of Y
    scale: float        # max of the two RMS radii


@dataclasses.dataclass
class Scales:
    x: float
    y: float
    xmean: np.ndarray
    ymean: np.ndarray


@dataclasses.dataclass
class Radius:
    x: float
    xmean: np.ndarray


def _centre(P):
    P = np.asarray(P, dtype=np.float64)
    m = P.mean(axis=0)
    C = P - m
    return C, m, float(np.sqrt(np.sum(C * C) / P.shape[0]))


def normalize(X, Y):
    Xc, xd, xs = _centre(X)
    Yc, yd, ys = _centre(Y)
    scale = xs if xs > ys else ys
    return Xc / scale, Yc / scale, Normal(xd, yd, scale)


def get_sd(X, Y) -> Scales:
    _, xd, xs = _centre(X)
    _, yd, ys = _centre(Y)
    return Scales(xs, ys, xd, yd)


def get_radius(X) -> Radius:
    _, xd, xs = _centre(X)
    return Radius(xs, xd)
