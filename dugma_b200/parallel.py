"""Multi-GPU use of the hot path: one process per GPU, torch.distributed for the plumbing.

Two ways the path divides (no collective is on the data path of either):
  * independent units — multistart poses of a problem, or whole problems — one per
    rank, nothing exchanged (bench.py --gpus N);
  * one large problem split by source rows: each rank evaluates its rows
    (dugma_energy_grad_range) and the partial energies and pose gradients (7 doubles in
    3D) are summed with one all-reduce; the surrogate coefficients likewise split by
    source and target rows (dugma_compi_range) and are summed with one all-reduce of 637
    (45 in 2D) doubles, and sigma's two partial sums (dugma_sigma_range) with one of 2.  Sums over rows are exactly the full sums up to FP64 rounding of
    the final additions.
"""
from __future__ import annotations

from typing import Callable, Sequence

import numpy as np


def row_ranges(n: int, world: int) -> list[tuple[int, int]]:
    """Contiguous, balanced source-row ranges for `world` ranks."""
    base, extra = divmod(n, world)
    out, i = [], 0
    for r in range(world):
        k = base + (1 if r < extra else 0)
        out.append((i, i + k))
        i += k
    return out


def energy_grad_sharded(n_rows: int, rank: int, world: int,
                        compute: Callable[[int, int], tuple[float, Sequence[float]]], group=None):
    """Sum of compute(i0, i1) over the ranks' row ranges; every rank returns (E, g).

    `compute` is the per-rank evaluation, normally
    lambda i0, i1: dugma_b200.api.energy_grad_range(handles, R, t, sig, i0, i1)."""
    import torch
    import torch.distributed as dist

    i0, i1 = row_ranges(n_rows, world)[rank]
    if i1 > i0:
        E, g = compute(i0, i1)
    else:
        E, g = 0.0, None
    g = np.zeros(0) if g is None else np.asarray(g, dtype=np.float64)
    ng = torch.tensor([g.size], dtype=torch.int64)
    if world > 1:
        dist.all_reduce(ng, op=dist.ReduceOp.MAX, group=group)
    buf = np.zeros(1 + int(ng.item()))
    buf[0] = E
    buf[1:1 + g.size] = g
    t = torch.from_numpy(buf)
    if world > 1:
        backend = dist.get_backend(group)
        if backend == "nccl":
            t = t.cuda()
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        t = t.cpu()
    out = t.numpy()
    return float(out[0]), out[1:].copy()


def _all_reduce_sum(vec: np.ndarray, world: int, group=None) -> np.ndarray:
    import torch
    import torch.distributed as dist
    t = torch.from_numpy(np.ascontiguousarray(vec, dtype=np.float64))
    if world > 1:
        if dist.get_backend(group) == "nccl":
            t = t.cuda()
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        t = t.cpu()
    return t.numpy().copy()


def compi_sharded(n_rows: int, m_rows: int, rank: int, world: int,
                  compute: Callable[[int, int, int, int], np.ndarray], n_coef: int, group=None) -> np.ndarray:
    """Surrogate coefficients summed over the ranks' source-row and target-row ranges.

    `compute(i0, i1, j0, j1)` is the per-rank evaluation, normally
    lambda i0, i1, j0, j1: dugma_b200.api.compi_range(handles, R, t, sig, i0, i1, j0, j1);
    every rank returns the full n_coef-vector."""
    i0, i1 = row_ranges(n_rows, world)[rank]
    j0, j1 = row_ranges(m_rows, world)[rank]
    part = np.zeros(n_coef)
    if i1 > i0 or j1 > j0:
        part = np.asarray(compute(i0, i1, j0, j1), dtype=np.float64).reshape(-1)[:n_coef]
    return _all_reduce_sum(part, world, group)


def sigma_sharded(n_rows: int, D: int, rank: int, world: int,
                  compute: Callable[[int, int], Sequence[float]], group=None) -> tuple[float, float]:
    """update_sig's sigma over source rows split across ranks: (quantised sigma as the reference
    returns it, unquantised sigma).  `compute(i0, i1)` returns the two partial sums of a row
    range, normally lambda i0, i1: dugma_b200.api.sigma_range(handles, R, t, i0, i1)."""
    i0, i1 = row_ranges(n_rows, world)[rank]
    part = np.zeros(2)
    if i1 > i0:
        part = np.asarray(compute(i0, i1), dtype=np.float64).reshape(-1)[:2]
    s0, s1 = _all_reduce_sum(part, world, group)
    return float(np.float32(s1 / 1e6 / n_rows)), float(s0 / (D * n_rows))
