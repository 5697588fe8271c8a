"""Wall-clock timing of the reference-interface plugin calls (update_sig, compi) through the C ABI.

    python -m dugma_b200.plugin_timing [--n 4096] [--reps 20]

On the 1K workload's generator (bumpy sphere, sensor covariances) at N = M = n: one init,
3 warm-up compi calls, `reps` timed compi calls, then `reps` timed update_sig calls, each a
host-to-host call like the reference's MEX gateway makes.  Prints one JSON line with the
medians in ms.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import api, synth


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=4096)
    ap.add_argument("--reps", type=int, default=20)
    a = ap.parse_args(argv)
    P = synth.workload0(n=a.n)
    _, h = api.init(P.X, P.X_C, P.Y, P.Y_C)
    try:
        R, t = P.R_G, P.t_G
        sig = api.update_sig(h, R, t)
        for _ in range(3):
            api.compi(h, R, t, sig=sig)
        tc = []
        for _ in range(a.reps):
            t0 = time.perf_counter()
            api.compi(h, R, t, sig=sig)
            tc.append(time.perf_counter() - t0)
        ts = []
        for _ in range(a.reps):
            t0 = time.perf_counter()
            api.update_sig(h, R, t)
            ts.append(time.perf_counter() - t0)
    finally:
        api.fr_m(h)
    print(json.dumps({"n": a.n, "compi_ms": 1e3 * float(np.median(tc)), "update_sig_ms": 1e3 * float(np.median(ts)),
                      "compi_pair_terms_per_s": a.n * a.n / float(np.median(tc))}), flush=True)


if __name__ == "__main__":
    main()
