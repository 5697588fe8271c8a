"""Golden fixtures: outputs of the reference's own plugins, recorded on a B200.

tests/golden/ref_*.npz were produced by tests/golden/make_golden.py, which runs the
reference's init.cu / update_sig.cu / compi.cu (compiled unmodified from the reference
sources by oracle/ref_build.py) on seeded inputs and stores inputs and outputs.  These
tests pin
  * the CPU oracle to the reference (no GPU needed), and
  * the CUDA library to the reference (marked gpu).
Tolerances: the reference inverts covariances and scales them in FP32 with fast-math
and forms each coefficient term in FP32 (compi.cu:800-3350), so
  coordinates       bit-exact
  inverse Sigma     |d| <= 2e-5 * max |block entry| per point
  |Sigma|^-1/2      relative 1e-6
  sigma             relative 3e-7 (the reference's FP32 conversion and tree sum)
  coefficients      max |dA| <= 1e-6 * max |A|
"""
import glob
import os

import numpy as np
import pytest

from oracle import oracle as orc

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "ref_*.npz")))


def _cm_blocks(a):
    return np.transpose(a, (0, 2, 1)).reshape(-1)


def _check_state(z, x, xinv_cm, wx, y, yinv_cm, wy):
    N, D = z["X"].shape
    M = z["Y"].shape[0]
    assert np.array_equal(x, z["d_X"]) and np.array_equal(y, z["d_Y"])
    for got, ref, n in ((xinv_cm, z["d_X_C"], N), (yinv_cm, z["d_Y_C"], M)):
        g, r = got.reshape(n, D * D), ref.reshape(n, D * D)
        scale = np.abs(r).max(axis=1, keepdims=True)
        assert np.all(np.abs(g - r) <= 2e-5 * scale)
    for got, ref in ((wx, z["det_X"]), (wy, z["det_Y"])):
        assert np.all(np.abs(got - ref) <= 1e-6 * np.abs(ref))
        assert np.array_equal(got == 0, ref == 0)


@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: os.path.basename(p)[4:-4])
def test_oracle_matches_reference_plugins(path):
    z = np.load(path)
    st = orc.State(z["X"], z["X_C"], z["Y"], z["Y_C"])
    D = z["X"].shape[1]
    _check_state(z, st.x.reshape(-1), _cm_blocks(st.xinv), st.wx, st.y.reshape(-1), _cm_blocks(st.yinv), st.wy)
    K = 637 if D == 3 else 45
    for k in range(len(z["sig"])):
        R, t = z["R"][k], z["t"][k]
        s = np.float32(st.sigma(R, t, quantised=True))
        assert abs(s - z["sig"][k]) <= 3e-7 * z["sig"][k]
        A = st.coef(R, t, float(z["sig"][k]))
        Ar = z["coef"][k]
        assert np.all(Ar[K:] == 0) and np.all(A[K:] == 0)
        assert np.abs(A[:K] - Ar[:K]).max() <= 1e-6 * np.abs(Ar[:K]).max()


def test_fixtures_present():
    assert len(FIXTURES) >= 3


@pytest.mark.gpu
@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: os.path.basename(p)[4:-4])
def test_library_matches_reference_plugins(path):
    import warnings

    from dugma_b200 import api
    from tests.test_gpu_parity import _read_state

    z = np.load(path)
    D = z["X"].shape[1]
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        _, h = api.init(z["X"], z["X_C"], z["Y"], z["Y_C"])
    try:
        s = _read_state(h)
        _check_state(z, s["x"], s["xinv"], s["wx"], s["y"], s["yinv"], s["wy"])
        K = 637 if D == 3 else 45
        for k in range(len(z["sig"])):
            R, t = z["R"][k], z["t"][k]
            sig = api.update_sig(h, R, t)
            assert abs(sig - z["sig"][k]) <= 3e-7 * z["sig"][k]
            A = api.compi(h, R, t, sig=float(z["sig"][k]))
            Ar = z["coef"][k][:K]
            assert np.abs(A - Ar).max() <= 1e-6 * np.abs(Ar).max()
    finally:
        api.fr_m(h)
