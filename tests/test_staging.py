"""Calls with and without the mapped pinned staging, and with and without programmatic dependent
launch between a call's kernels, give the same bits.

The plugin calls, the REF energy calls and the captured graphs hand the pose to their first
kernel (by value, or from the mapped staging for a graph) and read their results from the mapped
staging; without a mapped staging (DUGMA_NO_MAPPED_STAGING=1, read when a context is created)
the same kernels run with the pose copied to the device and the results copied back.  A child
process computes every entry point both ways is checked against bit for bit.
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import ctypes, json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from dugma_b200 import api, synth, _lib
from dugma_b200.pose import expmap
out = {}
for D, n in ((3, 1500), (2, 900)):
    if D == 3:
        P = synth.workload0(n=n)
        X, XC, Y, YC = P.X, P.X_C, P.Y, P.Y_C
        R, t = P.R_G @ expmap([0.03, -0.02, 0.01]), P.t_G + 0.01
    else:
        rng = np.random.default_rng(5)
        X = rng.standard_normal((n, 2)) * 0.5
        c, s = np.cos(0.2), np.sin(0.2)
        R = np.array([[c, -s], [s, c]])
        Y = (X - 0.05) @ R + rng.standard_normal((n, 2)) * 0.02
        A = rng.standard_normal((n, 2, 2)) * 0.1
        XC = A @ np.transpose(A, (0, 2, 1)) + 0.01 * np.eye(2)
        YC = XC[::-1].copy()
        t = np.array([0.05, -0.04])
    _, h = api.init(X, XC, Y, YC)
    sig = api.update_sig(h, R, t)
    A = api.compi(h, R, t, sig=sig)
    E0 = api.energy(h, R, t, sig)
    E, g, _ = api.energy_grad(h, R, t, sig)
    Eg, gg = api.energy_grad_range(h, R, t, sig, 3, n - 5)
    L = _lib.load()
    gr = ctypes.c_void_p()
    _lib.check(L.dugma_graph_create(h.arr, 0, ctypes.byref(gr)))
    dp = ctypes.POINTER(ctypes.c_double)
    Rc = np.ascontiguousarray(np.asarray(R).T); tt = np.ascontiguousarray(t, dtype=np.float64)
    Ev = ctypes.c_double(); gv = np.zeros(6)
    _lib.check(L.dugma_graph_eval(gr, Rc.ctypes.data_as(dp), tt.ctypes.data_as(dp), ctypes.c_double(sig),
                                  ctypes.byref(Ev), gv.ctypes.data_as(dp)))
    L.dugma_graph_destroy(gr)
    em = api.EMGraph(h)
    s_em, A_em = em(R, t)
    em.close()
    api.fr_m(h)
    out[str(D)] = {"sig": sig, "A": A.tolist(), "E0": E0, "E": E, "g": list(g), "Eg": Eg, "gg": list(gg),
                   "Ev": Ev.value, "gv": gv[:len(g)].tolist(), "s_em": s_em, "A_em": list(A_em)}
print(json.dumps(out))
"""


def _run(no_map: bool, no_pdl: bool = False):
    env = dict(os.environ)
    if no_map:
        env["DUGMA_NO_MAPPED_STAGING"] = "1"
    else:
        env.pop("DUGMA_NO_MAPPED_STAGING", None)
    if no_pdl:
        env["DUGMA_NO_PDL"] = "1"
    else:
        env.pop("DUGMA_NO_PDL", None)
    r = subprocess.run([sys.executable, "-c", CHILD, ROOT], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_mapped_and_copied_staging_give_the_same_bits():
    a, b = _run(False), _run(True)
    for D in ("3", "2"):
        for k in a[D]:
            assert np.array_equal(np.asarray(a[D][k]), np.asarray(b[D][k])), (D, k)
        # the graph and the single call agree as well
        assert a[D]["Ev"] == a[D]["E"] and np.array_equal(a[D]["gv"], a[D]["g"])
        assert a[D]["s_em"] == a[D]["sig"] and np.array_equal(a[D]["A_em"], a[D]["A"])


def test_dependent_launch_gives_the_same_bits():
    """The kernels of a call chained by programmatic dependent launch (the default) and launched one
    after the other (DUGMA_NO_PDL=1): every entry point, the captured graphs included, the same bits."""
    a, b = _run(False), _run(False, no_pdl=True)
    for D in ("3", "2"):
        for k in a[D]:
            assert np.array_equal(np.asarray(a[D][k]), np.asarray(b[D][k])), (D, k)
