"""Derive the 1-D refinement-factor-2 stencil coefficients and write
stencils_gen.h.

Every coefficient is an exact dyadic rational obtained from polynomial
interpolation (the method of CarpetX/stencils/stencils.jl:36-278):

* VC POLY p (odd p): Lagrange weights of the p+1 vertices i - (N/2 - 1),
  i = 0..p, evaluated at the midpoint x = 1/2 (coeffs1d<VC,POLY,p>,
  CarpetX/src/prolongate_3d_rf2_impl.hxx:59-99).
* CC POLY p: Lagrange weights of the cell centres i - N/2 evaluated at the
  left child x = -1/4 (impl.hxx:101-186).
* CC CONS p: weights giving the average over the left child [-1/2, 0] of the
  polynomial whose averages over the cells i - N/2 are the data, via the
  primitive interpolated at the N+1 cell faces (impl.hxx:237-314).
* CC ENO p, row m: the same conservative reconstruction on the cells
  i - (N/2 - shift), shift = m - p/2 (impl.hxx:316-384).

Run:  python gen_stencils.py  (rewrites stencils_gen.h next to this file)
"""
import os
from fractions import Fraction as F


def lagrange(nodes, k, x):
    r = F(1)
    for m, xm in enumerate(nodes):
        if m != k:
            r *= (x - xm) / (nodes[k] - xm)
    return r


def cons_weights(cells, xl, xh):
    faces = [F(cells[0]) - F(1, 2) + k for k in range(len(cells) + 1)]
    w = []
    for m in range(len(cells)):
        s = sum(lagrange(faces, k, xh) - lagrange(faces, k, xl) for k in range(m + 1, len(faces)))
        w.append(s / (xh - xl))
    return w


def vc_poly(p):
    N = p + 1
    i0 = N // 2 - 1
    nodes = [F(i - i0) for i in range(N)]
    return [lagrange(nodes, i, F(1, 2)) for i in range(N)]


def cc_poly(p):
    N = p + 1
    nodes = [F(i - N // 2) for i in range(N)]
    return [lagrange(nodes, i, F(-1, 4)) for i in range(N)]


def cc_cons(p):
    N = p + 1
    return cons_weights([i - N // 2 for i in range(N)], F(-1, 2), F(0))


def cc_eno(p, m):
    N = p + 1
    shift = m - p // 2
    return cons_weights([i - (N // 2 - shift) for i in range(N)], F(-1, 2), F(0))


def lit(q):
    assert q.denominator & (q.denominator - 1) == 0, "non-dyadic coefficient"
    return f"{q.numerator}.0 / {q.denominator}.0"


def arr(name, vals):
    # A constexpr function rather than an array, so that device code folds the
    # coefficient of an unrolled tap into an immediate operand.
    body = " : ".join(f"i == {i} ? {lit(v)}" for i, v in enumerate(vals)) + " : 0.0"
    return (f"CXB_HD constexpr double {name}(int i) {{ return {body}; }}\n"
            f"constexpr int {name}Len = {len(vals)};")


def main():
    out = ["// Generated by gen_stencils.py -- do not edit.",
           "// Exact dyadic 1-D prolongation weights (see gen_stencils.py for the",
           "// derivation); every value is exactly representable in FP64.",
           "#pragma once",
           "#if defined(__CUDACC__)",
           "#define CXB_HD __host__ __device__",
           "#else",
           "#define CXB_HD",
           "#endif",
           "namespace cxb {"]
    for p in (1, 3, 5, 7):
        out.append(arr(f"kVcPoly{p}", vc_poly(p)))
    for p in (1, 3, 5, 7):
        out.append(arr(f"kCcPoly{p}", cc_poly(p)))
    for p in range(0, 8):
        out.append(arr(f"kCcCons{p}", cc_cons(p)))
    for m in range(3):
        out.append(arr(f"kCcEno2Row{m}", cc_eno(2, m)))
    out.append("}  // namespace cxb")
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "stencils_gen.h")
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")


if __name__ == "__main__":
    main()
