"""The FP64 CPU oracle against itself and an independent numpy restatement.

These pin the oracle's formulas: the analytic pose gradient equals central
finite differences of the oracle energy, the C and numpy restatements of
P_ij agree, and the surrogate coefficients satisfy the defining identity
sum_k A_k b_k(dR, dt) = sum_ij P_ij q_ij(dR, dt) (energy3D.m:15-16,
compi.cu:699-791)."""
import numpy as np
import pytest

from oracle import oracle as orc
from dugma_b200 import synth
from dugma_b200.pose import expmap, rot2d


def small_problem(D=3, n=60, m=50, seed=0, bad=()):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((n, D)) * 0.5
    R0 = expmap(rng.standard_normal(3) * 0.3) if D == 3 else rot2d(0.4)
    Y = (X[np.arange(m) % n] - 0.1) @ R0 + rng.standard_normal((m, D)) * 0.05
    def covs(k):
        A = rng.standard_normal((k, D, D)) * 0.1
        return A @ np.transpose(A, (0, 2, 1)) + 0.01 * np.eye(D)
    XC, YC = covs(n), covs(m)
    for i in bad:
        XC[i] = np.diag([-1.0] + [1.0] * (D - 1))
    return X, XC, Y, YC


def fma32(a, b, c):
    """float32 fused multiply-add emulated in float64 (exact product, one rounding to float32
    after a float64 add; equal to the single-rounding fma except in rare double-rounding cases)."""
    return (a.astype(np.float64) * b.astype(np.float64) + c.astype(np.float64)).astype(np.float32)


def pose(D, seed=1):
    rng = np.random.default_rng(seed)
    if D == 3:
        return expmap(rng.standard_normal(3) * 0.2), rng.standard_normal(3) * 0.05
    return rot2d(0.15), rng.standard_normal(2) * 0.05


@pytest.mark.parametrize("D", [3, 2])
def test_prepare_matches_numpy_inverse(D):
    X, XC, Y, YC = small_problem(D, bad=(3, 7))
    inv, w, bad = orc.prepare(XC)
    assert bad == 2
    ref = np.linalg.inv(XC.astype(np.float32).astype(np.float64))
    ok = np.ones(len(XC), bool)
    ok[[3, 7]] = False
    np.testing.assert_allclose(inv[ok], ref[ok], rtol=1e-6, atol=0)
    assert np.all(inv[~ok] == 1e5) and np.all(w[~ok] == 0)
    np.testing.assert_allclose(w[ok], 1 / np.sqrt(np.linalg.det(XC[ok].astype(np.float32).astype(np.float64))), rtol=1e-6)


@pytest.mark.parametrize("D", [3, 2])
def test_energy_c_matches_numpy(D):
    X, XC, Y, YC = small_problem(D, bad=(5,))
    st = orc.State(X, XC, Y, YC)
    R, t = pose(D)
    E, g, _ = st.energy(R, t, 0.05)
    P = orc.np_pair_weights(st, R, t, 0.05)
    assert abs(E - P.sum()) <= 1e-12 * abs(E)


def _perturb(D, R, t, k, h):
    R2, t2 = R.copy(), t.copy()
    nr = 3 if D == 3 else 1
    if k < nr:
        w = np.zeros(3)
        if D == 3:
            w[k] = h
            R2 = expmap(w) @ R
        else:
            R2 = rot2d(h) @ R
    else:
        t2[k - nr] += h
    return R2, t2


@pytest.mark.parametrize("D", [3, 2])
@pytest.mark.parametrize("model", ["ref", "conv"])
def test_gradient_matches_central_fd(D, model):
    X, XC, Y, YC = small_problem(D)
    st = orc.State(X, XC, Y, YC)
    R, t = pose(D)
    f = st.energy if model == "ref" else st.energy_conv
    sig = 0.3 if model == "ref" else 0.05
    E, g, _ = f(R, t, sig)
    h = 1e-5
    fd = []
    for k in range(len(g)):
        Ep = f(*_perturb(D, R, t, k, h), sig)[0]
        Em = f(*_perturb(D, R, t, k, -h), sig)[0]
        fd.append((Ep - Em) / (2 * h))
    fd = np.array(fd)
    assert np.linalg.norm(fd - g) <= 1e-6 * np.linalg.norm(g), (g, fd)


@pytest.mark.parametrize("D", [3, 2])
@pytest.mark.parametrize("model", ["ref", "conv"])
def test_dEdx_matches_fd(D, model):
    X, XC, Y, YC = small_problem(D, n=20, m=25)
    st = orc.State(X, XC, Y, YC)
    R, t = pose(D)
    f = st.energy if model == "ref" else st.energy_conv
    E, g, dx = f(R, t, 0.2, with_dx=True)
    h = 1e-3
    for (i, a) in [(0, 0), (3, 1), (7, D - 1)]:
        Xp, Xm = X.copy(), X.copy()
        Xp[i, a] += h
        Xm[i, a] -= h
        # finite differences on the float32 state: perturb the stored coordinate exactly
        stp = orc.State(Xp, XC, Y, YC)
        stm = orc.State(Xm, XC, Y, YC)
        fp = (stp.energy if model == "ref" else stp.energy_conv)(R, t, 0.2)[0]
        fm = (stm.energy if model == "ref" else stm.energy_conv)(R, t, 0.2)[0]
        hh = float(stp.x[i, a]) - float(stm.x[i, a])
        assert abs((fp - fm) / hh - dx[i, a]) <= 1e-4 * np.abs(dx).max()


@pytest.mark.parametrize("D", [3, 2])
def test_coefficient_identity(D):
    """sum_k A_k b_k(dR, dt) equals sum_ij P_ij q_ij(dR, dt) at arbitrary (dR, dt)."""
    from dugma_b200.monomials import exponents
    X, XC, Y, YC = small_problem(D, n=30, m=40, bad=(2,))
    st = orc.State(X, XC, Y, YC)
    R, t = pose(D)
    A = st.coef(R, t, 0.3)
    K = 637 if D == 3 else 45
    assert np.all(A[K:] == 0)
    exps = exponents(D)
    rng = np.random.default_rng(3)
    for _ in range(3):
        if D == 3:
            dR = np.eye(3) + 0.2 * rng.standard_normal((3, 3))
            dt = 0.1 * rng.standard_normal(3)
        else:
            a, b = 1 + 0.1 * rng.standard_normal(), 0.2 * rng.standard_normal()
            dR = np.array([[a, -b], [b, a]])
            dt = 0.1 * rng.standard_normal(2)
        lhs = float(A[:K] @ orc.monomial_values(D, dR, dt, exps))
        rhs = orc.np_surrogate_direct(st, R, t, 0.3, dR, dt)
        assert abs(lhs - rhs) <= 1e-9 * abs(rhs)


@pytest.mark.parametrize("D", [3, 2])
def test_nn_matches_bruteforce_and_ties(D):
    X, XC, Y, YC = small_problem(D, n=80, m=70)
    Y[10] = Y[3]            # duplicate target: a tie that must resolve to the lower index
    st = orc.State(X, XC, Y, YC)
    R, t = pose(D)
    idx, d2 = st.nn(R, t, k=4)
    yp = (st.y.astype(np.float64) @ R.T + t).astype(np.float32)
    for i in range(0, len(X), 7):
        d = st.x[i] - yp
        dd = fma32(d[:, 1], d[:, 1], d[:, 0] * d[:, 0])
        if D == 3:
            dd = fma32(d[:, 2], d[:, 2], dd)
        order = np.lexsort((np.arange(len(dd)), dd))[:4]
        assert list(idx[i]) == list(order)
        assert np.array_equal(d2[i], dd[order])
    # the tie: whenever target 3 is a neighbour, 10 follows it and never precedes it
    for i in range(len(X)):
        r = list(idx[i])
        if 10 in r:
            assert 3 in r and r.index(3) < r.index(10)


def test_sigma_quantised_vs_exact():
    P = synth.workload0()
    st = orc.State(P.X, P.X_C, P.Y, P.Y_C)
    s_exact = st.sigma(np.eye(3), np.zeros(3), quantised=False)
    s_q = st.sigma(np.eye(3), np.zeros(3), quantised=True)
    assert abs(s_exact - s_q) <= 0.5e-6 + 1e-6 * s_exact
