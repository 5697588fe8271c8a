"""Rotation helpers shared by the host driver mirror and the tests.

Pose convention (as in the reference, DUGMA.m:75-80): the moving cloud Y is
mapped by y' = R y + t.  Gradients are taken with the left perturbation
R <- exp([w]x) R, t <- t + dt, so g = [dE/dw, dE/dt].
"""
from __future__ import annotations

import math

import numpy as np


def hat(w):
    return np.array([[0.0, -w[2], w[1]], [w[2], 0.0, -w[0]], [-w[1], w[0], 0.0]])


def expmap(w) -> np.ndarray:
    w = np.asarray(w, dtype=np.float64)
    th = float(np.linalg.norm(w))
    K = hat(w)
    if th < 1e-12:
        return np.eye(3) + K + 0.5 * K @ K
    return np.eye(3) + math.sin(th) / th * K + (1.0 - math.cos(th)) / (th * th) * (K @ K)


def logmap(R) -> np.ndarray:
    R = np.asarray(R, dtype=np.float64)
    c = max(-1.0, min(1.0, 0.5 * (np.trace(R) - 1.0)))
    th = math.acos(c)
    v = np.array([R[2, 1] - R[1, 2], R[0, 2] - R[2, 0], R[1, 0] - R[0, 1]])
    if th < 1e-8:
        return 0.5 * v
    if math.pi - th < 1e-6:
        w, V = np.linalg.eigh(0.5 * (R + R.T))
        axis = V[:, np.argmax(w)]
        return th * axis
    return th / (2.0 * math.sin(th)) * v


def rot2d(a: float) -> np.ndarray:
    return np.array([[math.cos(a), -math.sin(a)], [math.sin(a), math.cos(a)]])


def rotm2eul_zyx(R) -> np.ndarray:
    """ZYX Euler angles [z, y, x] in radians (the convention of MATLAB rotm2eul, DUGMA.m:80)."""
    R = np.asarray(R, dtype=np.float64)
    sy = -R[2, 0]
    sy = max(-1.0, min(1.0, sy))
    y = math.asin(sy)
    if abs(sy) < 1.0 - 1e-12:
        z = math.atan2(R[1, 0], R[0, 0])
        x = math.atan2(R[2, 1], R[2, 2])
    else:
        z = math.atan2(-R[0, 1], R[1, 1])
        x = 0.0
    return np.array([z, y, x])


def rotation_error_deg(R, R_G) -> float:
    return math.degrees(float(np.linalg.norm(logmap(np.asarray(R) @ np.asarray(R_G).T))))
