"""Generate the coefficient tables of the quadratic surrogate energy.

The reference's `compi` plugin returns, for a pose (R, t) and scale sigma, the
coefficients A_k of a polynomial Q(dR, dt) = sum_k A_k b_k(dR, dt) that
fmincon then minimises (DUGMA.m:60-73, energy3D.m:15-16, energy2D.m:7-8).
Symbolically, Q = sum_ij P_ij q_ij with

    q_ij(dR, dt) = e^T (dR C'_j dR^T) e + e^T B_i e,    e = x_i - dR y'_j - dt,

where y'_j = R y_j + t, C'_j = R (Sigma_y_j^-1 / sigma) R^T and
B_i = Sigma_x_i^-1 / sigma (compi.cu:699-791 computes exactly these per-pair
quantities).  In 3D dR is a general 3x3 matrix (12 unknowns with dt); in 2D
dR = [[r11, -r21], [r21, r11]] (energy2D.m, DUGMA.m:66).  Each A_k is
therefore sum_ij P_ij c_k(x_i, B_i, y'_j, C'_j) with c_k the coefficient of
the k-th monomial of q, in the monomial order of the `B = [...]` vectors of
energy3D.m / energy2D.m (that order is the output contract of `compi`).

This script derives c_k from q with sympy (it does not read the reference's
kernel source) and writes three generated headers:

  oracle/coef_terms.h            per-pair c_k in FP64 (the CPU oracle)
  dugma_b200/csrc/coef_map.h     c_k factored into i-side x j-side moments
  dugma_b200/csrc/monomials.h    exponent table of the monomials (surrogate)

The factorisation: every term of c_k is either (an entry of C'_j) x (a
y'-monomial of degree <= 2) x (an x-monomial of degree <= 2), or (an entry of
B_i) x (x-monomial) x (y'-monomial).  So A_k is a fixed linear combination of
the moments
    M1[psi, f] = sum_ij P_ij psi(C'_j, y'_j) f(x_i)     ("j-matrix" moments)
    M2[phi, g] = sum_ij P_ij phi(B_i, x_i) g(y'_j)       ("i-matrix" moments)
which the GPU accumulates as H1_j = sum_i P_ij f(x_i) and
H2_i = sum_j P_ij g(y'_j) (10 features each in 3D, 6 in 2D).

Run from the repository root:  python dugma_b200/gen/gen_coef.py [reference_dir]
The reference directory is read only for the monomial order.
"""
from __future__ import annotations

import os
import re
import sys
from fractions import Fraction

import sympy as sp

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), "..", ".."))


def sym_index(D):
    """Packed symmetric index order: diagonal first, then (0,1),(0,2),(1,2)."""
    if D == 3:
        return [(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)]
    return [(0, 0), (1, 1), (0, 1)]


def mono_list(D):
    """x-monomials of degree <= 2: 1, x_a, x_a x_b (a <= b, packed symmetric order)."""
    out = [()]
    out += [(a,) for a in range(D)]
    out += [tuple(sorted(p)) for p in sym_index(D)]
    return out


def parse_monomials(path, D):
    src = open(path).read()
    body = re.search(r"B\s*=\s*\[(.*?)\];", src, re.S).group(1)
    items = [s.strip() for s in body.split(",")]
    if D == 3:
        names = ["t1", "t2", "t3", "r11", "r12", "r13", "r21", "r22", "r23", "r31", "r32", "r33"]
    else:
        names = ["t1", "t2", "r11", "r21"]
    syms = {n: sp.Symbol(n) for n in names}
    mons = [sp.sympify(s.replace("^", "**"), locals=syms) for s in items]
    gens = [syms[n] for n in names]
    exps = [sp.Poly(m, *gens).monoms()[0] for m in mons]
    return names, gens, exps


def derive(D, ref_dir):
    names, gens, exps = parse_monomials(
        os.path.join(ref_dir, "energy3D.m" if D == 3 else "energy2D.m"), D)
    S = sym_index(D)
    x = sp.symbols(" ".join(f"x{a}" for a in range(D)))
    y = sp.symbols(" ".join(f"y{a}" for a in range(D)))
    Bs = sp.symbols(" ".join(f"B{a}{b}" for a, b in S))
    Cs = sp.symbols(" ".join(f"C{a}{b}" for a, b in S))

    def symmat(v):
        M = sp.zeros(D, D)
        for k, (a, b) in enumerate(S):
            M[a, b] = v[k]
            M[b, a] = v[k]
        return M

    Bm, Cm = symmat(Bs), symmat(Cs)
    g = dict(zip(names, gens))
    if D == 3:
        dR = sp.Matrix(3, 3, lambda r, c: g[f"r{r + 1}{c + 1}"])
        dt = sp.Matrix([g["t1"], g["t2"], g["t3"]])
    else:
        dR = sp.Matrix([[g["r11"], -g["r21"]], [g["r21"], g["r11"]]])
        dt = sp.Matrix([g["t1"], g["t2"]])
    xv, yv = sp.Matrix(x), sp.Matrix(y)
    e = xv - dR * yv - dt
    q = sp.expand((e.T * dR * Cm * dR.T * e)[0] + (e.T * Bm * e)[0])
    poly = sp.Poly(q, *gens)
    terms = dict(poly.terms())
    missing = set(terms) - set(exps)
    if missing:
        raise SystemExit(f"{D}D: q has monomials outside the reference order: {sorted(missing)[:5]}")
    coefs = [sp.expand(terms.get(ex, 0)) for ex in exps]

    # factor each coefficient into moment terms
    xm = mono_list(D)
    ym = mono_list(D)
    moments = {}      # key -> index; key = ('M1', c_idx, ymono, xmono) or ('M2', b_idx, xmono, ymono)
    cmap = []
    for ck in coefs:
        row = []
        for term in sp.Add.make_args(ck):
            if term == 0:
                continue
            coeff, rest = term.as_coeff_Mul()
            pw = rest.as_powers_dict()
            ci = [k for k, c in enumerate(Cs) if c in pw]
            bi = [k for k, b in enumerate(Bs) if b in pw]
            xe = tuple(sorted(sum(([a] * int(pw.get(x[a], 0)) for a in range(D)), [])))
            ye = tuple(sorted(sum(([a] * int(pw.get(y[a], 0)) for a in range(D)), [])))
            assert len(ci) + len(bi) == 1 and all(int(pw[s]) == 1 for s in [*(Cs[k] for k in ci), *(Bs[k] for k in bi)])
            if ci:
                key = ("M1", ci[0], ym.index(ye), xm.index(xe))
            else:
                key = ("M2", bi[0], xm.index(xe), ym.index(ye))
            if key not in moments:
                moments[key] = len(moments)
            row.append((moments[key], Fraction(int(coeff.p), int(coeff.q))))
        cmap.append(row)
    return dict(D=D, names=names, exps=exps, coefs=coefs, moments=moments, cmap=cmap,
                x=x, y=y, Bs=Bs, Cs=Cs)


def emit_oracle(res3, res2, path):
    out = ["/* Generated by dugma_b200/gen/gen_coef.py -- do not edit.",
           " * Oracle (test infrastructure): per-pair coefficients c_k(x, B, y', C') of the",
           " * monomials of q(dR, dt) = e^T dR C' dR^T e + e^T B e, e = x - dR y' - dt,",
           " * in the monomial order of energy3D.m:15 / energy2D.m:7 (the `compi` output",
           " * order, compi.cpp:47-64).  B and C' are packed symmetric (00,11,22,01,02,12). */",
           "#pragma once", ""]
    for res in (res3, res2):
        D = res["D"]
        K = len(res["coefs"])
        args = list(res["x"]) + list(res["Bs"]) + list(res["y"]) + list(res["Cs"])
        repl, red = sp.cse(res["coefs"], symbols=sp.numbered_symbols("w"))
        out.append(f"static inline void coef_terms_{D}d(const double* X, const double* B, "
                   f"const double* Y, const double* C, double* out /* [{K}] */)")
        out.append("{")
        for a in range(D):
            out.append(f"  const double x{a} = X[{a}], y{a} = Y[{a}];")
        for k, (a, b) in enumerate(sym_index(D)):
            out.append(f"  const double B{a}{b} = B[{k}], C{a}{b} = C[{k}];")
        for s, ex in repl:
            out.append(f"  const double {s} = {sp.ccode(ex)};")
        for k, ex in enumerate(red):
            out.append(f"  out[{k}] = {sp.ccode(ex)};")
        out.append("}")
        out.append("")
        del args
    open(path, "w").write("\n".join(out))


def emit_map(res3, res2, path):
    out = ["/* Generated by dugma_b200/gen/gen_coef.py -- do not edit.",
           " * Moment factorisation of the surrogate coefficients.  A moment is",
           " *   kind 1: M1 = sum_ij P_ij * Cp_j[m] * g_j[a] * f_i[b]   (Cp = C'_j packed entry m)",
           " *   kind 2: M2 = sum_ij P_ij * B_i[m]  * f_i[a] * g_j[b]",
           " * where f (x-monomials) and g (y'-monomials) run over 1, v_0..v_{D-1}, then the packed",
           " * symmetric products v_a v_b.  coef[k] = sum over its entries of num/den * moment. */",
           "#pragma once", "", "namespace dugma {", ""]
    for res in (res3, res2):
        D = res["D"]
        mom = sorted(res["moments"].items(), key=lambda kv: kv[1])
        out.append(f"constexpr int kNumMoments{D}D = {len(mom)};")
        out.append(f"constexpr int kNumCoef{D}D = {len(res['cmap'])};")
        out.append(f"/* kind, matrix entry m, a, b */")
        out.append(f"static const signed char kMoment{D}D[{len(mom)}][4] = {{")
        for (kind, m, a, b), idx in mom:
            out.append(f"  {{{1 if kind == 'M1' else 2}, {m}, {a}, {b}}},")
        out.append("};")
        flat = []
        start = [0]
        for row in res["cmap"]:
            for (mi, fr) in row:
                flat.append((mi, fr))
            start.append(len(flat))
        out.append(f"static const int kCoefStart{D}D[{len(start)}] = {{{', '.join(map(str, start))}}};")
        out.append(f"static const int kCoefMoment{D}D[{len(flat)}] = {{{', '.join(str(m) for m, _ in flat)}}};")
        out.append(f"static const double kCoefWeight{D}D[{len(flat)}] = {{{', '.join(f'{float(fr)!r}' for _, fr in flat)}}};")
        out.append("")
    out.append("}  // namespace dugma")
    open(path, "w").write("\n".join(out) + "\n")


def emit_monomials(res3, res2, path):
    out = ["/* Generated by dugma_b200/gen/gen_coef.py -- do not edit.",
           " * Exponents of the surrogate monomials b_k, in the order of energy3D.m:15",
           " * (variables t1 t2 t3 r11 r12 r13 r21 r22 r23 r31 r32 r33, row-major dR) and",
           " * energy2D.m:7 (variables t1 t2 r11 r21). */",
           "#pragma once", "", "namespace dugma {", ""]
    for res in (res3, res2):
        D = res["D"]
        nv = len(res["names"])
        out.append(f"static const unsigned char kMonoExp{D}D[{len(res['exps'])}][{nv}] = {{")
        for ex in res["exps"]:
            out.append("  {" + ", ".join(map(str, ex)) + "},")
        out.append("};")
        out.append("")
    out.append("}  // namespace dugma")
    open(path, "w").write("\n".join(out) + "\n")


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("DUGMA_REFERENCE", "")
    if not ref or not os.path.isdir(ref):
        raise SystemExit("usage: python -m dugma_b200.gen.gen_coef REFERENCE_TREE (or set DUGMA_REFERENCE)")
    res3 = derive(3, ref)
    res2 = derive(2, ref)
    for r in (res3, res2):
        print(f"{r['D']}D: {len(r['coefs'])} coefficients, {len(r['moments'])} moments, "
              f"{sum(len(c) for c in r['cmap'])} map entries")
    emit_oracle(res3, res2, os.path.join(ROOT, "oracle", "coef_terms.h"))
    emit_map(res3, res2, os.path.join(ROOT, "dugma_b200", "csrc", "coef_map.h"))
    emit_monomials(res3, res2, os.path.join(ROOT, "dugma_b200", "csrc", "monomials.h"))


if __name__ == "__main__":
    main()
