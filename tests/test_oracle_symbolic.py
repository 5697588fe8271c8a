"""Pin the oracle's coefficient expressions to the reference kernel source.

The oracle's per-pair coefficients c_k (oracle/coef_terms.h) and the GPU
moment map (dugma_b200/csrc/coef_map.h) are generated from the definition
q(dR, dt) = e^T dR C' dR^T e + e^T B e by dugma_b200/gen/gen_coef.py.  This
test parses the 637 (3D, compi.cu coef3D) and 45 (2D, compi.cu coef2D)
`temp = ...` expressions of the reference and checks each equals c_k
symbolically (with a_rc = C'_rc, b_rc = B_rc, m = y', n = x, symmetric
matrices).  It needs the reference tree and is skipped without it.
"""
import os
import re

import pytest

from oracle.ref_build import reference_tree

REF = reference_tree()
pytestmark = pytest.mark.skipif(REF is None, reason="reference tree not present (DUGMA_REFERENCE)")


def _ref_terms(body):
    return {int(m.group(1)): m.group(2) for m in re.finditer(r"i=(\d+);\s*temp=(.*?);\s*atomicAdd", body, re.S)}


@pytest.mark.parametrize("D", [3, 2])
def test_generated_coefficients_equal_reference_kernel(D):
    import sympy as sp
    from dugma_b200.gen import gen_coef

    res = gen_coef.derive(D, REF)
    src = open(os.path.join(REF, "compi.cu")).read()
    if D == 3:
        body = src[src.index("__global__ void coef3D(float *d_X,float *d_X_C,float *det_X,float *d_Y,"
                             "float *d_Y_C,float *det_Y,double *B_C)\n{"):]
    else:
        body = src[src.index("__global__ void coef2D"):src.index("__global__ void compi_redu")]
    terms = _ref_terms(body)
    K = 637 if D == 3 else 45
    assert sorted(terms) == list(range(K))
    S = gen_coef.sym_index(D)
    loc = {}
    for a in range(D):
        loc[f"n{a + 1}"] = res["x"][a]
        loc[f"m{a + 1}"] = res["y"][a]
    for k, (a, b) in enumerate(S):
        for (r, c) in ((a, b), (b, a)):
            loc[f"a{r + 1}{c + 1}"] = res["Cs"][k]
            loc[f"b{r + 1}{c + 1}"] = res["Bs"][k]
    for k in range(K):
        ref = sp.sympify(terms[k], locals=loc)
        assert sp.expand(ref - res["coefs"][k]) == 0, k
