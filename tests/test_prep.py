"""Scale helpers (normalize.m, get_sd*.m, get_radius.m) on the host."""
import numpy as np

from dugma_b200 import prep


def test_normalize_centres_and_scales_by_the_larger_radius():
    rng = np.random.default_rng(0)
    X = rng.standard_normal((50, 3)) * 2.0 + 5.0
    Y = rng.standard_normal((40, 3)) * 0.5 - 1.0
    Xn, Yn, nrm = prep.normalize(X, Y)
    assert np.allclose(Xn.mean(axis=0), 0, atol=1e-12) and np.allclose(Yn.mean(axis=0), 0, atol=1e-12)
    rx = np.sqrt(np.sum(Xn ** 2) / len(Xn))
    ry = np.sqrt(np.sum(Yn ** 2) / len(Yn))
    assert abs(max(rx, ry) - 1.0) <= 1e-12 and ry < rx
    assert np.allclose(Xn * nrm.scale + nrm.xd, X) and np.allclose(Yn * nrm.scale + nrm.yd, Y)


def test_sd_and_radius_agree_with_normalize():
    rng = np.random.default_rng(1)
    X, Y = rng.standard_normal((30, 2)), 3.0 * rng.standard_normal((20, 2))
    sd = prep.get_sd(X, Y)
    _, _, nrm = prep.normalize(X, Y)
    assert nrm.scale == max(sd.x, sd.y)
    r = prep.get_radius(Y)
    assert r.x == sd.y and np.array_equal(r.xmean, sd.ymean)
