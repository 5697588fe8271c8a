"""Monomial exponent tables of the surrogate energy (read from csrc/monomials.h).

Row k gives the exponents of b_k over (t1 t2 t3 r11 r12 r13 r21 r22 r23 r31 r32 r33)
in 3D and (t1 t2 r11 r21) in 2D, in the reference's order (energy3D.m:15, energy2D.m:7).
"""
from __future__ import annotations

import functools
import os
import re

import numpy as np

_HDR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "csrc", "monomials.h")


@functools.lru_cache(maxsize=None)
def exponents(D: int) -> np.ndarray:
    src = open(_HDR).read()
    body = re.search(r"kMonoExp%dD\[\d+\]\[\d+\] = \{(.*?)\};" % D, src, re.S).group(1)
    rows = re.findall(r"\{([^{}]*)\}", body)
    return np.array([[int(v) for v in r.split(",")] for r in rows], dtype=np.int64)


def surrogate(D: int, A, dR, dt) -> float:
    """Q(dR, dt) = sum_k A_k b_k(dR, dt) (energy3D.m:15-16 / energy2D.m:7-8)."""
    if D == 3:
        v = np.concatenate([np.asarray(dt, float), np.asarray(dR, float).reshape(-1)])
    else:
        v = np.array([dt[0], dt[1], dR[0][0], dR[1][0]], float)
    e = exponents(D)
    return float(np.asarray(A, float)[: e.shape[0]] @ np.prod(v[None, :] ** e, axis=1))
