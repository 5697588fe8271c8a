"""compi over all rows (the one-pass kernel) at ragged sizes.

The one-pass kernel's work grid -- source blocks per group and target tiles per chunk -- is
chosen per problem size, so every size below runs a different grid: single points, clouds
smaller than one 256-source block or one 32-target tile, sizes one past a block or tile
boundary, and clouds of very different sizes on the two sides.  Each result is checked against
the FP64 oracle (compi.cu:646-791 restated) at 2e-6 of the largest coefficient, repeated calls
must give the same bits, and a non-positive-definite covariance on each side (weight zero,
init.cu:48-57) must drop out.  A single pair is held to 2e-5: with one point per cloud, sigma
is that pair's own squared distance, so its exponent reaches ~100 (a weight of 2^-100) and the
FP32 rounding of the exponent -- the Cholesky form's z = U d and |z|^2, ~1e-7 of it -- is the
pair's error, with nothing to average it over (measured 1.06e-5 in 3D).
"""
import numpy as np
import pytest

from dugma_b200 import api
from oracle import oracle as orc
from tests.test_gpu_parity import _pose, _problem_small

pytestmark = pytest.mark.gpu

SIZES = [(1, 1), (3, 40), (40, 3), (257, 31), (255, 33), (1000, 4099), (3001, 777), (2048, 2048), (6000, 500),
         (500, 6000)]


@pytest.mark.parametrize("n,m", SIZES)
def test_compi_ragged_sizes_3d(n, m):
    _check(3, n, m, seed=n * 7 + m)


@pytest.mark.parametrize("n,m", [(1, 1), (257, 31), (3001, 777), (500, 6000)])
def test_compi_ragged_sizes_2d(n, m):
    _check(2, n, m, seed=n * 5 + m)


def _check(D, n, m, seed):
    bad = (0,) if min(n, m) > 1 else ()
    X, XC, Y, YC = _problem_small(D, n, m, seed=seed, bad=bad)
    R, t = _pose(D, seed=seed % 11, scale=0.1)
    import warnings
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        _, h = api.init(X, XC, Y, YC)
    try:
        sig = api.update_sig(h, R, t)
        A = api.compi(h, R, t, sig=sig)
        A2 = api.compi(h, R, t, sig=sig)
        assert np.array_equal(A, A2)
        Ao = orc.State(X, XC, Y, YC).coef(R, t, sig)[: A.size]
        scale = np.abs(Ao).max()
        assert scale > 0
        err = np.abs(A - Ao).max() / scale
        assert err <= (2e-5 if n * m == 1 else 2e-6), (n, m, err)
    finally:
        api.fr_m(h)


@pytest.mark.parametrize("side", ["sources", "targets"])
def test_every_covariance_of_one_cloud_neglected(side):
    """Every covariance of one cloud with det <= 0: all its weights are zero (init.cu:48-57), so
    every pair term vanishes -- compi's coefficients, the energy and its gradient are exactly
    zero, as in the oracle -- and the weight normaliser of that cloud (log2 of the largest
    weight, -inf here) must not turn into a NaN anywhere."""
    X, XC, Y, YC = _problem_small(3, 300, 280, seed=4)
    bad = np.diag([-1.0, 1.0, 1.0])
    if side == "sources":
        XC = np.repeat(bad[None], len(X), axis=0)
    else:
        YC = np.repeat(bad[None], len(Y), axis=0)
    R, t = _pose(3, seed=2, scale=0.1)
    import warnings
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        _, h = api.init(X, XC, Y, YC)
    try:
        sig = api.update_sig(h, R, t)
        assert np.isfinite(sig) and sig > 0
        A = api.compi(h, R, t, sig=sig)
        Ao = orc.State(X, XC, Y, YC).coef(R, t, sig)[: A.size]
        assert np.all(Ao == 0.0)
        assert np.all(A == 0.0)
        E, g, _ = api.energy_grad(h, R, t, sig)
        assert E == 0.0 and np.all(g == 0.0)
    finally:
        api.fr_m(h)
