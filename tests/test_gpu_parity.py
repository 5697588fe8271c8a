"""GPU parity: the CUDA path through the C ABI against the FP64 CPU oracle.

Tolerances (written per assertion):
  * init state (inverse covariances, |Sigma|^-1/2, FP32 coordinates): bit-exact;
  * nearest-neighbour indices and squared distances: bit-exact (same FP32 sequence);
  * sigma: bit-exact against the oracle's quantised and exact forms;
  * energy: relative 1e-6; pose gradient: relative 1e-5 (norm-wise), on the 1K sphere here,
    the 6K workload (noise-free source: 8-NN covariances of condition up to ~7e3) at three
    poses and three sigmas, the 64K harmonic surface and the 300K depth views in
    test_gpu_fullsize.py;
  * surrogate coefficients: |A - A_oracle| <= 2e-6 max|A_oracle|.
"""
import numpy as np
import pytest

from oracle import oracle as orc
from dugma_b200 import api, synth
from dugma_b200.pose import expmap, rot2d

pytestmark = pytest.mark.gpu


def _problem_small(D, n, m, seed=0, bad=(), dup=()):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((n, D)) * 0.5
    R0 = expmap(rng.standard_normal(3) * 0.3) if D == 3 else rot2d(0.4)
    Y = (X[np.arange(m) % n] - 0.1) @ R0 + rng.standard_normal((m, D)) * 0.05
    for (a, b) in dup:
        Y[a] = Y[b]

    def covs(k):
        A = rng.standard_normal((k, D, D)) * 0.1
        return A @ np.transpose(A, (0, 2, 1)) + 0.01 * np.eye(D)

    XC, YC = covs(n), covs(m)
    for i in bad:
        XC[i] = np.diag([-1.0] + [1.0] * (D - 1))
        if i < m:
            YC[i] = np.diag([1.0] * (D - 1) + [-2.0])
    return X, XC, Y, YC


def _pose(D, seed=1, scale=0.2):
    rng = np.random.default_rng(seed)
    if D == 3:
        return expmap(rng.standard_normal(3) * scale), rng.standard_normal(3) * 0.05
    return rot2d(scale), rng.standard_normal(2) * 0.05


def _rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def w0():
    P = synth.workload0()
    st = orc.State(P.X, P.X_C, P.Y, P.Y_C)
    _, h = api.init(P.X, P.X_C, P.Y, P.Y_C)
    yield P, st, h
    api.fr_m(h)


# ---------------------------------------------------------------- init
@pytest.mark.parametrize("D", [3, 2])
def test_init_state_bit_exact(D):
    X, XC, Y, YC = _problem_small(D, 300, 257, bad=(4, 9))
    st = orc.State(X, XC, Y, YC)
    with pytest.warns(UserWarning):
        _, h = api.init(X, XC, Y, YC)
    try:
        # read the six device buffers back through the library's own sizes
        got = _read_state(h)
        assert np.array_equal(got["x"], st.x.reshape(-1))
        assert np.array_equal(got["y"], st.y.reshape(-1))
        assert np.array_equal(got["xinv"], np.transpose(st.xinv, (0, 2, 1)).reshape(-1))
        assert np.array_equal(got["yinv"], np.transpose(st.yinv, (0, 2, 1)).reshape(-1))
        assert np.array_equal(got["wx"], st.wx)
        assert np.array_equal(got["wy"], st.wy)
        assert np.all(got["wx"][[4, 9]] == 0)
    finally:
        api.fr_m(h)


def _read_state(h):
    """Copy the six device buffers of a context back through torch (__cuda_array_interface__)."""
    import torch
    N, M, D = h.N, h.M, h.D
    sizes = {"x": N * D, "xinv": N * D * D, "y": M * D, "yinv": M * D * D, "wx": N, "wy": M}
    out = {}
    for k, (name, n) in enumerate(sizes.items()):
        out[name] = _device_f32(h.ptrs[k], n)
    return out


class _DevArray:
    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f4", "data": (ptr, False), "version": 3}


def _device_f32(ptr, n):
    import torch
    return torch.as_tensor(_DevArray(ptr, n), device="cuda").cpu().numpy().copy()


# ---------------------------------------------------------------- nearest neighbours / sigma
@pytest.mark.parametrize("D,k", [(3, 1), (3, 8), (2, 1), (2, 16)])
def test_nn_bit_exact_with_ties(D, k):
    X, XC, Y, YC = _problem_small(D, 1500, 1300, seed=3, dup=((700, 5), (1299, 5), (900, 901)))
    st = orc.State(X, XC, Y, YC)
    _, h = api.init(X, XC, Y, YC)
    try:
        R, t = _pose(D)
        idx, d2 = api.nn(h, R, t, k)
        oi, od = st.nn(R, t, k)
        assert np.array_equal(idx, oi)
        assert np.array_equal(d2, od)
    finally:
        api.fr_m(h)


def test_sigma_matches_oracle(w0):
    P, st, h = w0
    for (R, t) in [(np.eye(3), np.zeros(3)), _pose(3, 5)]:
        s_ref = api.update_sig(h, R, t)
        assert s_ref == np.float32(st.sigma(R, t, quantised=True))
        assert api.sigma(h, R, t) == st.sigma(R, t, quantised=False)
        # partial sums over an uneven partition of the rows (sharding update_sig): the quantised
        # terms add up exactly, the FP64 sums to rounding
        n = P.N
        parts = [api.sigma_range(h, R, t, a, b) for (a, b) in [(0, 1), (1, n // 3), (n // 3, n // 3), (n // 3, n)]]
        S = np.sum(parts, axis=0)
        assert np.float32(S[1] / 1e6 / n) == s_ref
        assert abs(S[0] / (3 * n) - st.sigma(R, t, quantised=False)) <= 1e-14 * S[0] / (3 * n)
    with pytest.raises(api.DugmaError):
        api.sigma_range(h, np.eye(3), np.zeros(3), 0, P.N + 1)


# ---------------------------------------------------------------- energy and adjoint
def _check_energy(h, st, R, t, sig, e_tol, g_tol):
    E, g, dx = api.energy_grad(h, R, t, sig, with_dx=True)
    Eo, go, dxo = st.energy(R, t, sig, with_dx=True)
    assert abs(E - Eo) <= e_tol * abs(Eo), (E, Eo)
    assert _rel(g, go) <= g_tol, (g, go)
    assert _rel(dx, dxo) <= g_tol * 10, _rel(dx, dxo)
    Ep = api.energy(h, R, t, sig)
    assert abs(Ep - Eo) <= e_tol * abs(Eo), (Ep, Eo)
    return E, g


def test_energy_adjoint_workload0(w0):
    P, st, h = w0
    R, t = P.R_G @ expmap([0.1, -0.2, 0.05]), P.t_G + 0.02
    sig = api.update_sig(h, R, t)
    _check_energy(h, st, R, t, sig, 1e-6, 1e-5)
    # the initial pose of a registration (identity), where sigma is large
    sig0 = api.update_sig(h, np.eye(3), np.zeros(3))
    _check_energy(h, st, np.eye(3), np.zeros(3), sig0, 1e-6, 1e-5)


@pytest.mark.parametrize("D", [3, 2])
@pytest.mark.parametrize("n,m", [(1, 1), (1, 300), (300, 1), (1025, 130), (77, 1031)])
def test_energy_adjoint_ragged_sizes(D, n, m):
    X, XC, Y, YC = _problem_small(D, n, m, seed=n + m, bad=(0,) if n > 2 and m > 2 else ())
    st = orc.State(X, XC, Y, YC)
    import warnings
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        _, h = api.init(X, XC, Y, YC)
    try:
        R, t = _pose(D, seed=7)
        _check_energy(h, st, R, t, 0.3, 1e-6, 1e-5)
    finally:
        api.fr_m(h)


@pytest.mark.parametrize("D", [3, 2])
@pytest.mark.parametrize("n,m", [(1, 1), (1, 300), (300, 1), (1025, 130), (77, 1031)])
def test_conv_and_knn_ragged_sizes_every_shape(D, n, m):
    """Ragged sizes (one source, one target, sizes off every tile and block multiple) through
    every compiled CONV adjoint / energy shape and every nearest-neighbour shape, k up to 16."""
    X, XC, Y, YC = _problem_small(D, n, m, seed=3 * n + m)
    st = orc.State(X, XC, Y, YC)
    _, h = api.init(X, XC, Y, YC)
    try:
        R, t = _pose(D, seed=11)
        Eo, go, dxo = st.energy_conv(R, t, 0.3, with_dx=True)
        for shape in api.shapes(3):
            api.set_shape(h, 3, shape)
            E, g, dx = api.energy_grad(h, R, t, 0.3, model=1, with_dx=True)
            assert abs(E - Eo) <= 1e-6 * abs(Eo), (shape, E, Eo)
            assert _rel(g, go) <= 1e-5, shape
            assert _rel(dx, dxo) <= 1e-4, shape
        for shape in api.shapes(4):
            api.set_shape(h, 4, shape)
            assert abs(api.energy(h, R, t, 0.3, model=1) - Eo) <= 1e-6 * abs(Eo), shape
        for shape in api.shapes(2):
            api.set_shape(h, 2, shape)
            for k in (1, 5, 9, 16):
                if k > m:
                    continue
                idx, d2 = api.nn(h, R, t, k)
                oi, od = st.nn(R, t, k)
                assert np.array_equal(idx, oi) and np.array_equal(d2, od), (shape, k)
    finally:
        api.fr_m(h)


@pytest.mark.parametrize("what", [0, 1, 3, 4])
@pytest.mark.parametrize("D", [3, 2])
def test_every_kernel_shape_matches_oracle(what, D):
    """Each compiled shape (REF scalar and packed f32x2 pair kernels: what 0 adjoint, 1 energy;
    CONV: 3 adjoint, 4 energy) against the oracle."""
    X, XC, Y, YC = _problem_small(D, 700, 1111, seed=21, bad=(3,))
    st = orc.State(X, XC, Y, YC)
    import warnings
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        _, h = api.init(X, XC, Y, YC)
    try:
        R, t = _pose(D, seed=8)
        model = 1 if what >= 3 else 0
        ref = st.energy_conv if model else st.energy
        Eo, go, dxo = ref(R, t, 0.2, with_dx=True)
        for shape in api.shapes(what):
            api.set_shape(h, what, shape)
            assert api.get_shape(h, what) == tuple(shape)
            if what in (0, 3):
                E, g, dx = api.energy_grad(h, R, t, 0.2, model=model, with_dx=True)
                assert _rel(g, go) <= 1e-5, shape
                assert _rel(dx, dxo) <= 1e-4, shape
            else:
                E = api.energy(h, R, t, 0.2, model=model)
            assert abs(E - Eo) <= 1e-6 * Eo, (shape, E, Eo)
    finally:
        api.fr_m(h)


@pytest.mark.parametrize("D", [3, 2])
def test_conv_model_matches_oracle(D):
    """CONV: per-pair combined covariance, its own determinant and inverse."""
    X, XC, Y, YC = _problem_small(D, 600, 777, seed=31)
    st = orc.State(X, XC, Y, YC)
    _, h = api.init(X, XC, Y, YC)
    try:
        R, t = _pose(D, seed=12)
        for sig in (0.05, 0.5):
            Eo, go, dxo = st.energy_conv(R, t, sig, with_dx=True)
            E, g, dx = api.energy_grad(h, R, t, sig, model=1, with_dx=True)
            assert abs(E - Eo) <= 1e-6 * Eo, (E, Eo)
            assert _rel(g, go) <= 1e-5, (g, go)
            assert _rel(dx, dxo) <= 1e-4
            assert abs(api.energy(h, R, t, sig, model=1) - Eo) <= 1e-6 * Eo
    finally:
        api.fr_m(h)


def test_conv_near_singular_pairs_use_fp64_inverse():
    """Nearly degenerate covariances on both sides: combined covariances of condition ~1e7."""
    rng = np.random.default_rng(5)
    n = 400
    X = rng.standard_normal((n, 3)) * 0.3
    Y = X + 1e-4 * rng.standard_normal((n, 3))
    v = np.array([1.0, 1.0, 1.0]) / np.sqrt(3.0)     # off-axis, so the matrices are far from diagonal
    XC = np.tile(np.eye(3) * 1e-9 + 1e-2 * np.outer(v, v), (n, 1, 1))
    YC = np.tile(np.eye(3) * 1e-9 + 1e-2 * np.outer(v, v), (n, 1, 1))
    # every other target well conditioned, so packed kernels meet packs with one rare half
    YC[1::2] = np.eye(3) * 1e-3
    st = orc.State(X, XC, Y, YC)
    _, h = api.init(X, XC, Y, YC)
    try:
        R, t = expmap([1e-3, -2e-3, 1e-3]), np.array([1e-4, 0.0, -1e-4])
        Eo, go, _ = st.energy_conv(R, t, 1.0)
        for shape in api.shapes(3):
            api.set_shape(h, 3, shape)
            E, g, _ = api.energy_grad(h, R, t, 1.0, model=1)
            print(f"near-singular CONV {shape}: energy rel err {abs(E - Eo) / Eo:.3e}, grad rel err {_rel(g, go):.3e}")
            assert abs(E - Eo) <= 1e-5 * Eo, shape
            assert _rel(g, go) <= 1e-4, shape
    finally:
        api.fr_m(h)


@pytest.mark.parametrize("D", [3, 2])
def test_conv_few_near_singular_targets(D):
    """A handful of near-singular targets among thousands: most tiles of the packed CONV kernels
    stay on the straight-line fast path, a few are redone exactly from the sums saved at their
    start, so the saved sums must carry over correctly between fast and redone tiles."""
    rng = np.random.default_rng(17)
    n, m = 700, 3001
    X = rng.standard_normal((n, D)) * 0.4
    Y = X[rng.integers(0, n, m)] + 0.02 * rng.standard_normal((m, D))
    v = np.ones(D) / np.sqrt(D)
    XC = np.tile(np.eye(D) * 2e-3, (n, 1, 1))
    YC = np.tile(np.eye(D) * 2e-3, (m, 1, 1))
    rare = np.array([5, 6, 1000, 2047, 2999])
    # rank-one plus a tiny floor, on both sides of the pairs it meets: near-singular combined
    # covariances for the sources that are degenerate along the same direction
    YC[rare] = np.eye(D) * 1e-10 + 1e-2 * np.outer(v, v)
    XC[:40] = np.eye(D) * 1e-10 + 1e-2 * np.outer(v, v)
    st = orc.State(X, XC, Y, YC)
    _, h = api.init(X, XC, Y, YC)
    try:
        R, t = _pose(D, seed=4, scale=0.05)
        for sig in (0.3, 1.0):
            Eo, go, dxo = st.energy_conv(R, t, sig, with_dx=True)
            for shape in api.shapes(3):
                api.set_shape(h, 3, shape)
                E, g, dx = api.energy_grad(h, R, t, sig, model=1, with_dx=True)
                assert abs(E - Eo) <= 1e-5 * Eo, (shape, E, Eo)
                assert _rel(g, go) <= 1e-4, shape
                assert _rel(dx, dxo) <= 1e-3, shape
            for shape in api.shapes(4):
                api.set_shape(h, 4, shape)
                assert abs(api.energy(h, R, t, sig, model=1) - Eo) <= 1e-5 * Eo, shape
    finally:
        api.fr_m(h)


@pytest.fixture(scope="module")
def w1():
    P = synth.workload1()
    st = orc.State(P.X, P.X_C, P.Y, P.Y_C)
    _, h = api.init(P.X, P.X_C, P.Y, P.Y_C)
    yield P, st, h
    api.fr_m(h)


def _w1_pose(P, k):
    # near convergence (small sigma), the ground truth, and a pose farther out
    return [(P.R_G @ expmap([0.05, 0.1, -0.05]), P.t_G * 0.95), (P.R_G, P.t_G),
            (P.R_G @ expmap([0.3, -0.2, 0.1]), P.t_G + 0.05)][k]


@pytest.mark.parametrize("k", [0, 1, 2])
@pytest.mark.parametrize("sig_mult", [1.0, 4.0, 16.0])
def test_energy_adjoint_workload1_ill_conditioned(w1, k, sig_mult):
    """The 6K workload (source covariances of condition up to ~7e3) inside the precision
    contract: energy 1e-6 and pose gradient 1e-5 relative to the FP64 oracle, at the sigma that
    update_sig gives for the pose and at 4x and 16x that sigma (wider kernels: more pairs
    with large, ill-conditioned quadratic forms)."""
    P, st, h = w1
    R, t = _w1_pose(P, k)
    sig = api.update_sig(h, R, t) * sig_mult
    E, g, _ = api.energy_grad(h, R, t, sig)
    Eo, go, _ = st.energy(R, t, sig)
    print(f"workload1 pose {k} sig x{sig_mult:g}: energy rel err {abs(E - Eo) / Eo:.3e}, "
          f"grad rel err {_rel(g, go):.3e}")
    assert abs(E - Eo) <= 1e-6 * Eo
    assert _rel(g, go) <= 1e-5


def _oracle_fd(st, R, t, sig, h):
    """Central finite differences of the FP64 oracle's energy over [omega, t] (left perturbation)."""
    g = np.zeros(6)
    for q in range(6):
        Es = []
        for sgn in (1.0, -1.0):
            if q < 3:
                w = np.zeros(3)
                w[q] = sgn * h
                Es.append(st.energy(expmap(w) @ R, t, sig)[0])
            else:
                t2 = np.array(t, float)
                t2[q - 3] += sgn * h
                Es.append(st.energy(R, t2, sig)[0])
        g[q] = (Es[0] - Es[1]) / (2.0 * h)
    return g


def test_fd_grad_workload1(w1):
    """The 6K workload against central finite differences.  The plain form (library energies,
    step 1e-4) agrees with the FP64 oracle's central differences of the same step.  That step is
    coarse here: the narrowest source Gaussians are ~3.5e-5 wide (largest eigenvalue of s
    Sigma_x^-1 ~8e8), so the step-1e-4 difference carries an O(h^2) truncation error of ~1.4e-2.
    The fused adjoint is therefore checked against the oracle's differences extrapolated to zero
    step (Richardson on steps 2e-6 and 1e-6, error O(h^4))."""
    P, st, h = w1
    R, t = _w1_pose(P, 0)
    sig = api.update_sig(h, R, t)
    E, g, _ = api.energy_grad(h, R, t, sig)
    Efd, gfd = api.energy_fd_grad(h, R, t, sig, step=1e-4)
    go_fd4 = _oracle_fd(st, R, t, sig, 1e-4)
    go_lim = (4.0 * _oracle_fd(st, R, t, sig, 1e-6) - _oracle_fd(st, R, t, sig, 2e-6)) / 3.0
    print(f"workload1 FD: plain form vs oracle (step 1e-4) {_rel(gfd, go_fd4):.3e}; adjoint vs oracle "
          f"extrapolated {_rel(g, go_lim):.3e}; adjoint vs step-1e-4 differences {_rel(g, go_fd4):.3e}")
    assert abs(Efd - E) <= 1e-6 * E
    assert _rel(gfd, go_fd4) <= 1e-4
    assert _rel(g, go_lim) <= 1e-5


@pytest.mark.parametrize("side", ["sources", "targets"])
@pytest.mark.parametrize("D", [3, 2])
def test_indefinite_inverse_uses_horner_form(D, side):
    """A few covariances with det > 0 that are not positive definite (the reference accepts them:
    only det <= 0 is neglected, init.cu:48-57), on the source or on the target side: no Cholesky
    factor exists, so the packed adjoint (sources) and compi (either side) run on the Horner form;
    the energy, its gradient and the coefficients still match the oracle."""
    X, XC, Y, YC = _problem_small(D, 300, 260, seed=9)
    # det > 0 with two negative eigenvalues; their quadratic forms stay small (|exponent| < 1)
    C = XC if side == "sources" else YC
    C[3] = np.diag([-100.0, -100.0, 0.01]) if D == 3 else np.diag([-100.0, -100.0])
    C[77] = C[3]
    st = orc.State(X, XC, Y, YC)
    _, h = api.init(X, XC, Y, YC)
    try:
        R, t = _pose(D, seed=5, scale=0.1)
        for sig in (0.05, 0.5):
            Eo, go, _ = st.energy(R, t, sig)
            E, g, _ = api.energy_grad(h, R, t, sig)
            assert np.isfinite(Eo)
            assert abs(E - Eo) <= 1e-6 * abs(Eo), (E, Eo)
            assert _rel(g, go) <= 1e-5
            assert abs(api.energy(h, R, t, sig) - Eo) <= 1e-6 * abs(Eo)
            A = api.compi(h, R, t, sig=sig)
            Ao = st.coef(R, t, sig)[: A.size]
            assert np.abs(A - Ao).max() <= 2e-6 * np.abs(Ao).max()
    finally:
        api.fr_m(h)


def test_sigma_extremes(w0):
    P, st, h = w0
    R, t = _pose(3, 11)
    for sig in (1e-7, 1e-3, 10.0, 1e4):
        E, g, _ = api.energy_grad(h, R, t, sig)
        Eo, go, _ = st.energy(R, t, sig)
        assert np.isfinite(E) and np.all(np.isfinite(g))
        if Eo > 0:
            assert abs(E - Eo) <= 1e-6 * Eo + 1e-300
        else:
            assert E == 0


def test_fd_grad_plain_form(w0):
    P, st, h = w0
    R, t = P.R_G @ expmap([0.2, 0.1, 0.0]), P.t_G
    sig = 0.05
    E, g = api.energy_fd_grad(h, R, t, sig, step=1e-4)
    Eo, go, _ = st.energy(R, t, sig)
    assert abs(E - Eo) <= 1e-6 * Eo
    assert _rel(g, go) <= 1e-4


@pytest.mark.parametrize("D", [3, 2])
@pytest.mark.parametrize("n,m", [(1, 1), (700, 1111), (1025, 130)])
def test_ref_precision_model_matches_oracle(D, n, m):
    """The FP64 per-pair (reference precision) energy: FP64 sums in another order only, so
    relative 1e-11; its gradient is the central-difference plain form, compared with the
    oracle's central differences over the same perturbations (left rotation exp(h e_q) R,
    then t + h e_q; relative 1e-7); asking it for an adjoint is an argument error."""
    X, XC, Y, YC = _problem_small(D, n, m, seed=5 + n, bad=(2,) if n > 2 and m > 2 else ())
    st = orc.State(X, XC, Y, YC)
    import warnings
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        _, h = api.init(X, XC, Y, YC)
    try:
        R, t = _pose(D, seed=9)
        for sig in (0.05, 0.4):
            Eo, go, _ = st.energy(R, t, sig)
            E = api.energy(h, R, t, sig, model=2)
            assert abs(E - Eo) <= 1e-11 * abs(Eo) + 1e-300, (E, Eo)
        hstep = 1e-4
        Ef, gf = api.energy_fd_grad(h, R, t, 0.4, step=hstep, model=2)
        Eo, go, _ = st.energy(R, t, 0.4)
        assert abs(Ef - Eo) <= 1e-11 * abs(Eo) + 1e-300
        nr = 3 if D == 3 else 1
        gfd = []
        for q in range(nr + D):
            ev = []
            for sgn in (1.0, -1.0):
                R2, t2 = R.copy(), np.array(t, dtype=float)
                if q < nr:
                    w = np.zeros(3)
                    w[q] = sgn * hstep
                    R2 = (expmap(w) if D == 3 else rot2d(sgn * hstep)) @ R
                else:
                    t2[q - nr] += sgn * hstep
                ev.append(st.energy(R2, t2, 0.4)[0])
            gfd.append((ev[0] - ev[1]) / (2 * hstep))
        assert _rel(gf, gfd) <= 1e-7, (gf, gfd)
        assert _rel(gf, go) <= 1e-3   # central-difference truncation against the analytic gradient
        with pytest.raises(api.DugmaError):
            api.energy_grad(h, R, t, 0.4, model=2)
    finally:
        api.fr_m(h)


def test_bounded_wait_gives_up_and_device_stays_usable(w0):
    """The failure path of every tile wait, made to happen: a wait on an mbarrier that nothing
    completes gives up after its poll limit and reports a timeout instead of hanging; the
    device and an existing context keep working afterwards."""
    import ctypes
    from dugma_b200 import _lib
    L = _lib.load()
    flag = ctypes.c_int(0)
    assert L.dugma_wait_selftest(1000, ctypes.byref(flag)) == 0
    assert flag.value == 1
    assert L.dugma_wait_selftest(0, ctypes.byref(flag)) == _lib.ERR_ARG
    P, st, h = w0
    R, t = _pose(3, 31)
    E, g, _ = api.energy_grad(h, R, t, 0.05)
    Eo, go, _ = st.energy(R, t, 0.05)
    assert abs(E - Eo) <= 1e-6 * Eo and _rel(g, go) <= 1e-5


def test_range_partials_sum_to_total(w0):
    P, st, h = w0
    R, t = _pose(3, 2)
    E, g, _ = api.energy_grad(h, R, t, 0.05)
    parts = [api.energy_grad_range(h, R, t, 0.05, a, b) for (a, b) in [(0, 333), (333, 334), (334, 1000)]]
    assert abs(sum(p[0] for p in parts) - E) <= 1e-12 * E
    assert _rel(sum(p[1] for p in parts), g) <= 1e-12


def test_results_deterministic(w0):
    P, st, h = w0
    R, t = _pose(3, 4)
    a = api.energy_grad(h, R, t, 0.05)
    b = api.energy_grad(h, R, t, 0.05)
    assert a[0] == b[0] and np.array_equal(a[1], b[1])


def test_graph_replay_matches_eager(w0):
    P, st, h = w0
    gr = api.Graph(h)
    try:
        for s in range(3):
            R, t = _pose(3, 20 + s)
            E1, g1 = gr(R, t, 0.05)
            E2, g2, _ = api.energy_grad(h, R, t, 0.05)
            assert E1 == E2 and np.array_equal(g1, g2)
    finally:
        gr.close()


def test_autotune_keeps_results(w0):
    P, st, h = w0
    R, t = _pose(3, 9)
    rep = api.autotune(h, 0)
    assert "ms" in rep
    E, g, _ = api.energy_grad(h, R, t, 0.05)
    Eo, go, _ = st.energy(R, t, 0.05)
    assert abs(E - Eo) <= 1e-6 * Eo and _rel(g, go) <= 1e-5


# ---------------------------------------------------------------- coefficients (compi)
@pytest.mark.parametrize("D", [3, 2])
def test_compi_coefficients(D):
    if D == 3:
        P = synth.workload0()
        X, XC, Y, YC = P.X, P.X_C, P.Y, P.Y_C
        R, t = P.R_G @ expmap([0.1, 0.0, -0.1]), P.t_G
    else:
        X, XC, Y, YC = _problem_small(2, 700, 650, seed=5, bad=(3,))
        R, t = _pose(2)
    st = orc.State(X, XC, Y, YC)
    import warnings
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        _, h = api.init(X, XC, Y, YC)
    try:
        sig = api.update_sig(h, R, t)
        A = api.compi(h, R, t, sig=sig)
        Ao = st.coef(R, t, sig)[: A.size]
        err = np.abs(A - Ao).max() / np.abs(Ao).max()
        print(f"{D}D coefficients: max |dA| / max |A| = {err:.3e}")
        assert err <= 2e-6
        # partial coefficients over a 3-way partition of the source rows and an uneven
        # 2-way partition of the target rows add up to the whole (sharding across GPUs)
        n, m = X.shape[0], Y.shape[0]
        parts = [api.compi_range(h, R, t, sig, 0, n // 3, 0, m // 4),
                 api.compi_range(h, R, t, sig, n // 3, n // 2, m // 4, m),
                 api.compi_range(h, R, t, sig, n // 2, n, m, m)]
        S = np.sum(parts, axis=0)
        assert np.abs(S - A).max() <= 1e-6 * np.abs(A).max()
        assert np.abs(api.compi_range(h, R, t, sig, 0, n, 0, m) - A).max() <= 1e-12 * np.abs(A).max()
        with pytest.raises(api.DugmaError):
            api.compi_range(h, R, t, sig, 0, n + 1, 0, m)
    finally:
        api.fr_m(h)


# ---------------------------------------------------------------- data preparation
def test_knn_covariance_matches_cpu_estimator():
    """GPU k-NN sample covariance (k = 8, eigenvalues clamped) against the seeded generators'
    scipy-based estimator; neighbour sets can differ only on near-ties, so compare the bulk."""
    rng = np.random.default_rng(9)
    pts = synth.bumpy_sphere(rng, 3000)
    ref = synth._knn_sample_cov(pts, 1e-6, 1e-2)
    got = api.knn_covariance(pts, k=8, lo=1e-6, hi=1e-2)
    err = np.abs(got - ref).reshape(len(pts), -1).max(axis=1) / np.abs(ref).reshape(len(pts), -1).max(axis=1)
    assert np.mean(err < 1e-6) > 0.99, np.sort(err)[-10:]
    assert np.all(np.linalg.eigvalsh(got) >= 1e-6 * (1 - 1e-9))


# ---------------------------------------------------------------- the reference's C++ entry points
def test_reference_cpp_entry_points_match_python_mirror(tmp_path):
    """A C++ program calls init / cpd (update_sig) / cpd (compi) / fr_m by the reference's own
    signatures, as its MEX gateways do; the results equal the C-ABI path's (same kernels)."""
    import subprocess
    from tests.test_abi import build_mex_harness
    exe = build_mex_harness(tmp_path)
    P = synth.workload0(n=700)
    R, t = P.R_G @ expmap([0.05, 0.02, -0.03]), P.t_G
    inp, out = str(tmp_path / "in.bin"), str(tmp_path / "out.bin")
    with open(inp, "wb") as f:
        np.array([P.N, P.M, 3], np.int32).tofile(f)
        for a in (P.X, np.transpose(P.X_C, (0, 2, 1)), P.Y, np.transpose(P.Y_C, (0, 2, 1)), np.asarray(R).T,
                  np.asarray(t)):
            np.ascontiguousarray(a, np.float64).tofile(f)
    subprocess.run([exe, inp, out], check=True, timeout=300)
    res = np.fromfile(out, np.float64)
    assert res[0] == 1.0
    _, h = api.init(P.X, P.X_C, P.Y, P.Y_C)
    try:
        sig = api.update_sig(h, R, t)
        A = api.compi(h, R, t, sig=sig)
    finally:
        api.fr_m(h)
    assert res[1] == sig
    assert np.array_equal(res[2:2 + 637], A)


@pytest.mark.parametrize("D", [3, 2])
def test_em_graph_step_equals_update_sig_then_compi(D):
    """One captured EM step (update_sig at a pose, then compi at that pose and sigma, sigma kept
    on the device) gives what the two plugin calls give, bit for bit, over several poses (the
    registration loop uses it; tests/test_kinect.py holds that loop to the recorded poses)."""
    X, XC, Y, YC = _problem_small(D, 700, 650, seed=21)
    _, h = api.init(X, XC, Y, YC)
    g = api.EMGraph(h)
    try:
        for seed in range(4):
            R, t = _pose(D, seed=seed, scale=0.15)
            sig_g, A_g = g(R, t)
            sig = api.update_sig(h, R, t)
            A = api.compi(h, R, t, sig=sig)
            assert sig_g == sig
            assert np.array_equal(A_g, A)
    finally:
        g.close()
        api.fr_m(h)


def test_conv_ill_conditioned_without_cancellation_stays_accurate():
    """The CONV model's FP64 redo is triggered by det < 1e-6 x (product of the diagonal) of the
    combined covariance, the cancellation that the FP32 adjugate and determinant suffer, not by
    the condition number itself.  Here every combined covariance has condition ~1e7 but its thin
    direction is the z axis and the pose rotates about z, so the matrices stay block diagonal:
    det equals the product of the diagonal up to the well-conditioned 2 x 2 block, no entry of
    the adjugate cancels, and the FP32 path meets the contract (energy 1e-6, gradient 1e-5)."""
    rng = np.random.default_rng(31)
    n, m = 600, 700
    X = np.zeros((n, 3))
    X[:, :2] = rng.uniform(-1, 1, (n, 2))
    Y = X[rng.integers(0, n, m)].copy()
    Y[:, :2] += 0.03 * rng.standard_normal((m, 2))
    Y[:, 2] += 3e-5 * rng.standard_normal(m)          # |d_z|^2 comparable with the thin variance
    XC = np.tile(np.diag([1e-2, 1e-2, 1e-9]), (n, 1, 1))
    YC = np.tile(np.diag([1e-2, 1e-2, 1e-9]), (m, 1, 1))
    st = orc.State(X, XC, Y, YC)
    _, h = api.init(X, XC, Y, YC)
    try:
        c, s_ = np.cos(0.2), np.sin(0.2)
        R = np.array([[c, -s_, 0], [s_, c, 0], [0, 0, 1.0]])
        t = np.array([0.01, -0.02, 0.0])
        for sig in (0.5, 1.0):
            Eo, go, _ = st.energy_conv(R, t, sig)
            E, g, _ = api.energy_grad(h, R, t, sig, model=1)
            assert abs(E - Eo) <= 1e-6 * Eo, (sig, E, Eo)
            assert _rel(g, go) <= 1e-5, sig
    finally:
        api.fr_m(h)
