"""compi's one pass with the source-side sums on the tensor cores (coef_tc_kernel: tcgen05.mma of
kind::tf32, p in tensor memory, the targets' monomials in shared memory, the three-term TF32
split) against the FP64 oracle and against the default one-pass kernel (FP32 pipe only).

The kernel is chosen when a context is created (DUGMA_COEF_KERNEL = 1: one source per thread,
four blocks per SM), so a child process computes the
coefficients with it on ragged sizes in 3D and 2D -- clouds smaller than one 128-source M-block,
one past a tile boundary, more rows than fit one round of work items -- twice each (the repeat must
give the same bits).  The problems are those of test_compi_sizes.py (same seeds).  The parent holds
them to the oracle at the tolerance of the other compi tests (2e-6 of the largest coefficient; the
single pair 2e-5, its exponent ~100) and to the default kernel's coefficients at 4e-6.  (A single
pair whose exponent falls below FP32's range, -126 in log2, is 0 in both kernels and tiny in the
FP64 oracle; these seeds stay inside it.)
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from dugma_b200 import api
from oracle import oracle as orc
from tests.test_gpu_parity import _pose, _problem_small

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CASES = [(3, 1, 1), (3, 257, 31), (3, 3001, 777), (3, 2048, 2048), (3, 500, 6000), (2, 257, 31), (2, 3000, 2500)]

CHILD = r"""
import json, sys, warnings
import numpy as np
sys.path.insert(0, sys.argv[1])
from dugma_b200 import api
from tests.test_gpu_parity import _pose, _problem_small
out = []
for D, n, m in json.loads(sys.argv[2]):
    bad = (0,) if min(n, m) > 1 else ()
    X, XC, Y, YC = _problem_small(D, n, m, seed=n * 7 + m, bad=bad)
    R, t = _pose(D, seed=(n * 7 + m) % 11, scale=0.1)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        _, h = api.init(X, XC, Y, YC)
    sig = api.update_sig(h, R, t)
    A = api.compi(h, R, t, sig=sig)
    A2 = api.compi(h, R, t, sig=sig)
    api.fr_m(h)
    out.append({"sig": sig, "A": A.tolist(), "same": bool(np.array_equal(A, A2))})
print(json.dumps(out))
"""


def _child(kind):
    env = dict(os.environ, DUGMA_COEF_KERNEL=str(kind))
    r = subprocess.run([sys.executable, "-c", CHILD, ROOT, json.dumps(CASES)], env=env, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


@pytest.mark.parametrize("kind", [1])
def test_tensor_core_compi_matches_oracle_and_default_kernel(kind):
    res = _child(kind)
    import warnings
    for (D, n, m), r in zip(CASES, res):
        bad = (0,) if min(n, m) > 1 else ()
        X, XC, Y, YC = _problem_small(D, n, m, seed=n * 7 + m, bad=bad)
        R, t = _pose(D, seed=(n * 7 + m) % 11, scale=0.1)
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")
            _, h = api.init(X, XC, Y, YC)
        try:
            sig = api.update_sig(h, R, t)
            A0 = api.compi(h, R, t, sig=sig)   # the default kernel (FP32 pipe)
        finally:
            api.fr_m(h)
        assert r["sig"] == sig and r["same"], (D, n, m)
        A = np.asarray(r["A"])
        Ao = orc.State(X, XC, Y, YC).coef(R, t, sig)[: A.size]
        scale = np.abs(Ao).max()
        err = np.abs(A - Ao).max() / scale
        err0 = np.abs(A - A0).max() / scale
        print(f"kind {kind} D {D} {n}x{m}: vs oracle {err:.2e}, vs default kernel {err0:.2e}")
        assert err <= (2e-5 if n * m == 1 else 2e-6), (D, n, m, err)
        assert err0 <= 4e-6, (D, n, m, err0)
