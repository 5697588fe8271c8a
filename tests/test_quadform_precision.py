"""Why compi evaluates its quadratic forms in the Cholesky form (CPU, no device).

Each pair's two exponents are quadratic forms d^T B d of a source matrix B_i = s Sigma_x_i^-1 and a
target matrix C'_j = R (s Sigma_y_j^-1) R^T, held in FP32.  In the Horner form the FP32 rounding of
the matrix entries moves d^T B d by up to ~cond(B) ulps; in the Cholesky form |U d|^2 (U^T U = B,
U rounded) it moves by ~sqrt(cond(B)) ulps.  On the reference's ill-conditioned golden case
(tests/golden/ref_illcond2048.npz: 8-NN sample covariances, condition up to 1e4) this check rounds
only the matrices to FP32 -- everything else in FP64 -- and compares the energy and its first
moment sum_ij P_ij d_ij with the exact ones: the Cholesky form's error is at least 5x smaller.
"""
import os

import numpy as np

FIX = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_illcond2048.npz")


def _moments(qb, qc, W, d):
    P = W * (np.exp(-0.5 * qc) + np.exp(-0.5 * qb))
    return P.sum(), (P[..., None] * d).sum((0, 1))


def _errors():
    z = np.load(FIX)
    X, XC, Y, YC = z["X"], z["X_C"], z["Y"], z["Y_C"]
    R, t, sig = z["R"][0], z["t"][0], float(z["sig"][0])
    s = 1.0 / sig
    B = s * np.linalg.inv(XC)                                        # per source
    C = s * np.einsum("ab,nbc,dc->nad", R, np.linalg.inv(YC), R)     # per target
    d = X[:, None, :] - (Y @ R.T + t)[None, :, :]
    W = (1 / np.sqrt(np.linalg.det(XC)))[:, None] * (1 / np.sqrt(np.linalg.det(YC)))[None, :]
    f32 = lambda M: M.astype(np.float32).astype(np.float64)   # noqa: E731  (exact arithmetic after)
    qB = lambda M: np.einsum("ija,iab,ijb->ij", d, M, d, optimize=True)   # noqa: E731
    qC = lambda M: np.einsum("ija,jab,ijb->ij", d, M, d, optimize=True)   # noqa: E731
    UB = f32(np.swapaxes(np.linalg.cholesky(B), -1, -2))
    UC = f32(np.swapaxes(np.linalg.cholesky(C), -1, -2))
    zB = np.einsum("iab,ijb->ija", UB, d, optimize=True)
    zC = np.einsum("jab,ijb->ija", UC, d, optimize=True)
    E0, g0 = _moments(qB(B), qC(C), W, d)
    Eh, gh = _moments(qB(f32(B)), qC(f32(C)), W, d)
    Ec, gc = _moments((zB * zB).sum(-1), (zC * zC).sum(-1), W, d)
    rel = lambda a, b: np.abs(a - b).max() / np.abs(b).max()   # noqa: E731
    return rel(Eh, E0), rel(gh, g0), rel(Ec, E0), rel(gc, g0), np.linalg.cond(XC).max()


def test_cholesky_form_is_the_accurate_one_on_ill_conditioned_covariances():
    eh, gh, ec, gc, cond = _errors()
    print(f"condition up to {cond:.1e}: Horner energy {eh:.2e} moment {gh:.2e}; "
          f"Cholesky energy {ec:.2e} moment {gc:.2e}")
    assert cond > 1e3
    assert ec * 5 <= eh and gc * 5 <= gh
    assert gc <= 5e-7
