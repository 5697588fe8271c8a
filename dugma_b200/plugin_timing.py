"""Wall-clock timing of the reference-interface plugin calls (update_sig, compi) through the C ABI.

    python -m dugma_b200.plugin_timing [--n 4096] [--reps 20] [--knn K] [--nn K]

On the 1K workload's generator (bumpy sphere, sensor covariances) at N = M = n: one init,
3 warm-up compi calls, `reps` timed compi calls, then `reps` timed update_sig calls, each a
host-to-host call like the reference's MEX gateway makes.  With --knn K it also times the
k-nearest-neighbour covariance estimator (dugma_knn_covariance) on the source cloud.  With
--nn K it also reports the device time of the k-nearest-neighbour search kernels behind
dugma_nn (CUDA events recorded by the library, `dugma_timing`), averaged over `reps` calls.
Prints one JSON line with the medians in ms.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import time

import numpy as np

from . import _lib, api, synth


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=4096)
    ap.add_argument("--reps", type=int, default=20)
    ap.add_argument("--knn", type=int, default=0, help="also time the k-NN covariance estimator with this k")
    ap.add_argument("--nn", type=int, default=0, help="also time the k-nearest-neighbour kernels with this k")
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
        if a.nn:
            L = _lib.load()
            api.nn(h, R, t, a.nn)
            _lib.check(L.dugma_timing(h.arr, 1, None, None))
            for _ in range(a.reps):
                api.nn(h, R, t, a.nn)
            ms = ctypes.c_double(0)
            nl = ctypes.c_int(0)
            _lib.check(L.dugma_timing(h.arr, 2, ctypes.byref(ms), ctypes.byref(nl)))
            _lib.check(L.dugma_timing(h.arr, 0, None, None))
            nn_ms = ms.value / a.reps
    finally:
        api.fr_m(h)
    line = {"n": a.n, "compi_ms": 1e3 * float(np.median(tc)), "update_sig_ms": 1e3 * float(np.median(ts)),
            "compi_pair_terms_per_s": a.n * a.n / float(np.median(tc))}
    if a.knn:
        api.knn_covariance(P.X, k=a.knn)
        tk = []
        for _ in range(max(1, a.reps // 4)):
            t0 = time.perf_counter()
            api.knn_covariance(P.X, k=a.knn)
            tk.append(time.perf_counter() - t0)
        line["knn_covariance_ms"] = 1e3 * float(np.median(tk))
        line["knn_k"] = a.knn
    if a.nn:
        line.update({"nn_k": a.nn, "nn_kernel_ms": nn_ms, "nn_pairs_per_s": a.n * a.n / (nn_ms * 1e-3)})
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
