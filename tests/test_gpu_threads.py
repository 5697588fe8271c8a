"""Concurrent use from several host threads: each thread creates its own contexts, evaluates
(update_sig, energy and pose gradient, compi, 8 nearest neighbours) and frees them, while the
others do the same.  Contexts share the library's caches (device arenas, pinned staging,
streams, moment tables); every result must equal the single-threaded one bit for bit (all
reductions run in a fixed order)."""
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from dugma_b200 import api, synth
from dugma_b200.pose import expmap

pytestmark = pytest.mark.gpu


def _run(trial, rounds):
    P = synth.workload0(trial=trial, n=1500 + 97 * trial)
    R = P.R_G @ expmap([0.04, -0.02, 0.03 * (trial + 1)])
    t = P.t_G + 0.01
    out = []
    for _ in range(rounds):
        _, h = api.init(P.X, P.X_C, P.Y, P.Y_C)
        try:
            sig = api.update_sig(h, R, t)
            E, g, _ = api.energy_grad(h, R, t, sig)
            A = api.compi(h, R, t, sig=sig)
            idx, d2 = api.nn(h, R, t, 8)
            out.append((sig, E, g.copy(), A.copy(), idx.copy(), d2.copy()))
        finally:
            api.fr_m(h)
    return out


def _same(a, b):
    return all(np.array_equal(np.asarray(x), np.asarray(y)) for x, y in zip(a, b))


def test_threads_with_own_contexts_match_single_thread():
    trials = [0, 1, 2, 3]
    ref = {k: _run(k, 1)[0] for k in trials}
    with ThreadPoolExecutor(max_workers=len(trials)) as ex:
        futs = {k: ex.submit(_run, k, 6) for k in trials}
        res = {k: f.result(timeout=600) for k, f in futs.items()}
    for k in trials:
        for r in res[k]:
            assert _same(r, ref[k]), f"thread for trial {k} differs from the single-threaded result"
