"""compi's one-pass work grid (dugma_coef_work_grid: the host-side model that picks source
blocks per group and target tiles per chunk).  No device work.

Invariants at every size: the groups cover every 256-source block and the chunks every
32-target tile, no group or chunk is empty, at most 64 copies of either side and at most 16 GB
of them.  Regimes measured on the B200 (444 resident blocks): small clouds run one round of
items (every block busy at once), large ones about 4-5 rounds of items (dynamic balancing); the
grids the model picks at 4096 and 64K are the ones measured fastest there.
"""
import ctypes
import math

import pytest

from dugma_b200 import _lib

RESIDENT = 148 * 3


def _grid(N, M, resident=RESIDENT):
    g = (ctypes.c_int * 4)()
    _lib.check(_lib.load().dugma_coef_work_grid(N, M, resident, g))
    return tuple(g)


@pytest.mark.parametrize("N,M", [(1, 1), (255, 257), (1000, 1000), (4096, 4096), (6000, 6000), (16384, 16384),
                                 (65536, 65536), (300000, 300000), (3000000, 3000000), (500, 200000),
                                 (200000, 500)])
def test_grid_covers_the_problem(N, M):
    SB, n_grp, jt, n_jc = _grid(N, M)
    n_ib = math.ceil(N / 256)
    tiles = math.ceil(M / 128) * 128 // 32
    assert n_grp * SB >= n_ib and (n_grp - 1) * SB < n_ib
    assert n_jc * jt >= tiles and (n_jc - 1) * jt < tiles
    assert 1 <= n_grp <= 64 and 1 <= n_jc <= 64
    assert (n_jc * N + n_grp * M) * 128 <= 16e9 or (n_grp == 1 and n_jc == 1)


def test_regimes():
    # 4096: one round of items (the fastest of the grids measured there: 16 x 26)
    SB, n_grp, jt, n_jc = _grid(4096, 4096)
    assert (SB, n_grp, jt, n_jc) == (1, 16, 5, 26) and n_grp * n_jc <= RESIDENT
    # 64K: several rounds of items of a few hundred tiles
    SB, n_grp, jt, n_jc = _grid(65536, 65536)
    assert n_grp * n_jc >= 4 * RESIDENT and 100 <= SB * jt <= 400
    # a full round of items even at 3M points (the copy cap allows it)
    SB, n_grp, jt, n_jc = _grid(3000000, 3000000)
    assert n_grp * n_jc >= 0.9 * RESIDENT


def test_bad_arguments():
    g = (ctypes.c_int * 4)()
    assert _lib.load().dugma_coef_work_grid(0, 10, RESIDENT, g) == _lib.ERR_ARG
    assert _lib.load().dugma_coef_work_grid(10, 10, 0, g) == _lib.ERR_ARG
