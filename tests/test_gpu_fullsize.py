"""GPU parity at the workloads' full sizes (65536 x 65536 harmonic surface, 300000-point depth
views), where the FP64 oracle cannot evaluate every pair in a test's time.  Checked instead:

  * sampled source rows against the oracle (the oracle evaluates those rows against all
    targets): energy relative 1e-6, pose gradient relative 1e-5 (the library's
    dugma_energy_grad_range over the same rows), each with a floor of 1e-24 of the whole
    evaluation's value: per-pair terms more than 2^-126 below the largest weight product
    flush to zero in FP32 (the oracle keeps them in FP64), which can matter only for a row
    range whose whole contribution is that far below the total;
  * nearest neighbours of sampled rows bit-exact (the oracle's search of those rows);
  * the 256 sources with the nearest targets (they carry the energy when sigma is small) as
    a problem of their own against all targets: energy 1e-6, gradient 1e-5, no floor;
  * size-independent properties of the full evaluation: the sum of row-range partials over a
    partition equals the whole (FP64 rounding of the final additions, 1e-12), and two
    evaluations give identical bits (fixed-order reductions);
  * compi (the surrogate coefficients) over all rows, one pass over the pairs, against the sum
    of row-range partials computed by the other kernels (one coefficient pass per side) over an
    uneven partition of both clouds: 1e-6 of the largest coefficient (the two add the FP32
    per-pair terms in different orders), and two calls give identical bits.
"""
import numpy as np
import pytest

from oracle import oracle as orc
from dugma_b200 import api, synth
from dugma_b200.pose import expmap

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _check_full(P, R, t, rows, k_nn=1):
    _, h = api.init(P.X, P.X_C, P.Y, P.Y_C)
    try:
        sig = api.update_sig(h, R, t)
        E, g, _ = api.energy_grad(h, R, t, sig)
        # determinism
        E2, g2, _ = api.energy_grad(h, R, t, sig)
        assert E == E2 and np.array_equal(g, g2)
        # partition of the rows into uneven ranges
        n = P.N
        cuts = [0, 1, n // 7, n // 2, n - 3, n]
        parts = [api.energy_grad_range(h, R, t, sig, a, b) for a, b in zip(cuts, cuts[1:])]
        assert abs(sum(p[0] for p in parts) - E) <= 1e-12 * abs(E)
        assert _rel(sum(p[1] for p in parts), g) <= 1e-12
        # sampled rows against the oracle
        st = orc.State(P.X, P.X_C, P.Y, P.Y_C)
        for (a, b) in rows:
            Eg, gg = api.energy_grad_range(h, R, t, sig, a, b)
            Eo, go, _ = st.energy(R, t, sig, i0=a, i1=b)
            print(f"rows [{a}, {b}): E {Eo:.3e} of {E:.3e}, energy rel err {abs(Eg - Eo) / abs(Eo):.2e}, "
                  f"grad rel err {_rel(gg, go):.2e}")
            assert abs(Eg - Eo) <= 1e-6 * abs(Eo) + 1e-24 * abs(E), (a, b, Eg, Eo)
            assert np.linalg.norm(gg - go) <= 1e-5 * np.linalg.norm(go) + 1e-24 * np.linalg.norm(g), (a, b, gg, go)
        # nearest neighbours of sampled rows, bit-exact
        idx, d2 = api.nn(h, R, t, k_nn)
        for (a, b) in rows:
            sub = orc.State(P.X[a:b], P.X_C[a:b], P.Y, P.Y_C)
            oi, od = sub.nn(R, t, k_nn)
            assert np.array_equal(idx[a:b], oi) and np.array_equal(d2[a:b], od)
        # the sources that carry the energy (nearest targets closest) against all targets,
        # as a problem of their own on the GPU and in the oracle
        sel = np.sort(np.argsort(d2[:, 0], kind="stable")[:256])
        _, hs = api.init(P.X[sel], P.X_C[sel], P.Y, P.Y_C)
        try:
            Es, gs, _ = api.energy_grad(hs, R, t, sig)
        finally:
            api.fr_m(hs)
        Eo, go, _ = orc.State(P.X[sel], P.X_C[sel], P.Y, P.Y_C).energy(R, t, sig)
        print(f"256 nearest rows: E {Eo:.3e} of {E:.3e}, energy rel err {abs(Es - Eo) / abs(Eo):.2e}, "
              f"grad rel err {_rel(gs, go):.2e}")
        assert abs(Eo) >= 1e-3 * abs(E)        # they do carry the energy
        assert abs(Es - Eo) <= 1e-6 * abs(Eo)
        assert _rel(gs, go) <= 1e-5
        # compi: one pass over all pairs against the per-side passes over a partition
        A = api.compi(h, R, t, sig=sig)
        assert np.array_equal(A, api.compi(h, R, t, sig=sig))
        m = P.M
        ci, cj = [0, n // 3, n], [0, m // 5, m]
        S = sum(api.compi_range(h, R, t, sig, ci[k], ci[k + 1], cj[k], cj[k + 1]) for k in range(2))
        err = np.abs(S - A).max() / np.abs(A).max()
        print(f"compi: one pass against the per-side passes, max |dA| / max |A| = {err:.2e}")
        assert err <= 1e-6
    finally:
        api.fr_m(h)


def test_harmonic_surface_65536():
    P = synth.workload2()
    R, t = P.R_G @ expmap([0.004, -0.002, 0.003]), P.t_G + 0.001
    _check_full(P, R, t, rows=[(0, 256), (40000, 40256), (65536 - 256, 65536)], k_nn=8)


def test_depth_views_300000():
    P = synth.workload4()
    R, t = P.R_G @ expmap([0.02, 0.01, -0.02]), P.t_G + 0.005
    _check_full(P, R, t, rows=[(0, 128), (150000, 150128), (P.N - 128, P.N)])
