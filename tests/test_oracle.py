"""CPU tests of the oracle: the C restatement (oracle/cx_oracle.c) against the
reference's own outputs (golden fixtures generated by the reference operators,
and the reference build itself when present), and the reference's own
known-answer checks (test_interp1d, CarpetX/src/prolongate_3d_rf2_impl.hxx:
882-1174) restated."""
import hashlib
import importlib.util
import os

import numpy as np
import pytest

from helpers import ALL_OPS, FAMILIES, assert_bitwise, box_shape, random_case, region_mask
from config1 import config1_case

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "prolong_golden.npz")


def golden_cases():
    z = np.load(GOLDEN)
    n = len([k for k in z.files if k.endswith("_meta")])
    for i in range(n):
        key = f"{i:04d}"
        m = z[key + "_meta"]
        yield dict(typ=str(z[key + "_type"]), order=int(m[0]), it=int(m[1]), pg=int(m[2]),
                   ncomp=int(m[3]), clo=tuple(m[4:7]), chi=tuple(m[7:10]), flo=tuple(m[10:13]),
                   fhi=tuple(m[13:16]), rlo=tuple(m[16:19]), rhi=tuple(m[19:22]),
                   crse=z[key + "_crse"], fine=z[key + "_fine"])


def test_golden_covers_every_operator():
    seen = {(c["typ"], c["order"], c["it"]) for c in golden_cases()}
    assert seen == set(ALL_OPS)


def test_oracle_matches_golden(cx):
    for c in golden_cases():
        fine = np.full_like(c["fine"], np.nan)
        cx.prolong(c["typ"], c["order"], c["it"], c["pg"], c["crse"], c["clo"], c["chi"], fine,
                   c["flo"], c["fhi"], c["rlo"], c["rhi"], c["ncomp"])
        m = region_mask(c["flo"], c["fhi"], c["rlo"], c["rhi"])
        assert_bitwise(fine[:, m], c["fine"][:, m], f"{c['typ']} o{c['order']} it{c['it']}")


def test_oracle_matches_reference_random(cx, ref):
    rng = np.random.default_rng(7)
    for kind in ("normal", "jumps", "ties"):
        for typ, order, it in ALL_OPS:
            for pg in (0, 1):
                c = random_case(rng, ref, typ, order, it, ncomp=int(rng.integers(1, 4)),
                                max_n=10, kind=kind)
                f1 = np.full((c["ncomp"],) + box_shape(c["flo"], c["fhi"]), np.nan)
                f2 = f1.copy()
                args = (c["crse"], c["clo"], c["chi"])
                ref.prolong(typ, order, it, pg, *args, f1, c["flo"], c["fhi"], c["rlo"], c["rhi"],
                            c["ncomp"])
                cx.prolong(typ, order, it, pg, *args, f2, c["flo"], c["fhi"], c["rlo"], c["rhi"],
                           c["ncomp"])
                assert_bitwise(f2, f1, f"{typ} o{order} it{it} pg{pg} {kind}")


def test_oracle_config1_checksum(cx):
    c = config1_case()
    fine = np.zeros((1,) + box_shape(c["flo"], c["fhi"]))
    cx.prolong("interpolate", 3, 0, 0, c["crse"], c["clo"], c["chi"], fine, c["flo"], c["fhi"],
               c["flo"], c["fhi"], 1)
    want = open(os.path.join(HERE, "golden", "config1_sha256.txt")).read().strip()
    assert hashlib.sha256(np.ascontiguousarray(fine).tobytes()).hexdigest() == want


def _load_generator():
    path = os.path.join(HERE, "..", "carpetx_b200", "csrc", "gen_stencils.py")
    spec = importlib.util.spec_from_file_location("gen_stencils", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_product_coefficients_match_oracle(cx):
    """The product's coefficient derivation (gen_stencils.py) and the oracle's
    (cx_oracle.c, int128 rationals) are independent; both must agree."""
    g = _load_generator()
    for p in (1, 3, 5, 7):
        assert np.array_equal(cx.coeffs(0, 0, p), [float(v) for v in g.vc_poly(p)])
        assert np.array_equal(cx.coeffs(1, 0, p), [float(v) for v in g.cc_poly(p)])
    for p in range(8):
        assert np.array_equal(cx.coeffs(1, 2, p), [float(v) for v in g.cc_cons(p)])
    for m in range(3):
        assert np.array_equal(cx.coeffs(1, 3, 2, m), [float(v) for v in g.cc_eno(2, m)])


# 1-D stencil kinds per (family, order, centring) as (intp, order) -- used to
# build exact polynomial data for the reproduction test
def dir_stencil(typ, order, cent):
    vc = cent == 0
    if typ == "interpolate":
        return ("poly", order)
    if typ == "conservative":
        return ("vccons" if vc else "cons", order if vc else (0 if order == 0 else 2))
    if typ == "ddf":
        return ("poly", order) if vc else ("cons", order - 1)
    if typ in ("eno", "poly-eno3lfb"):
        if vc:
            return ("poly", order)
        return ("cons", 0) if order == 1 else ("eno", 2)
    if typ == "minmod":
        return ("poly", order) if vc else ("minmod", 1)
    if typ in ("hermite", "natural"):
        return ("poly", order) if vc else ("cons", order)
    if typ == "poly-cons3lfb":
        return ("poly", order) if vc else ("cons", min(order, 3))
    raise ValueError(typ)


def poly_line(cent, intp, q, lo, n):
    """Coarse data along one direction for x^q (vertex: point values at x = i;
    cell POLY: values at cell centres i + 1/2; cell CONS/ENO/MINMOD: cell
    averages, as test_interp1d builds them, impl.hxx:896-913, 988-1017) and
    the exact fine values.  Small integers/dyadics: every operation exact."""
    i = np.arange(lo, lo + n, dtype=float)
    if cent == 0 or intp == "poly":
        xs = i + 0.5 * cent
        return xs ** q
    fint = lambda x: x ** (q + 1)  # noqa: E731
    return fint(i + 1.0) - fint(i)


def fine_exact(cent, intp, q, lo, n):
    f = np.arange(lo, lo + n, dtype=float)
    if cent == 0:
        return (f / 2) ** q
    if intp == "poly":
        return (f / 2 + 0.25) ** q
    # average over the fine cell [f/2, f/2 + 1/2] of (q+1) x^q
    fint = lambda x: x ** (q + 1)  # noqa: E731
    return (fint(f / 2 + 0.5) - fint(f / 2)) * 2


def reproduction_cases():
    """(family, order, indextype, direction, q): exact reproduction of x^q,
    q <= the stencil order, for data varying along one direction only
    (test_interp1d, impl.hxx:885-975 and 977-1039; minmod reproduces linear
    data, :1115-1174; ENO: every shift reproduces order-2 averages,
    :1051-1113)."""
    out = []
    for typ, orders in FAMILIES.items():
        for order in orders:
            for it in range(8):
                if typ == "conservative" and order == 0 and it != 7:
                    # deprecated VC CONS 0 writes 0 at odd fine vertices
                    # (empty stencil, impl.hxx:225, 619-628): no reproduction
                    continue
                for d in range(3):
                    cent = (it >> (2 - d)) & 1
                    intp, p = dir_stencil(typ, order, cent)
                    for q in range(p + 1):
                        out.append((typ, order, it, d, q))
    return out


def make_reproduction(oracle, typ, order, it, d, q, n=6):
    cent = (it >> (2 - d)) & 1
    intp, p = dir_stencil(typ, order, cent)
    flo = [4, 4, 4]
    fhi = [4 + n - 1] * 3
    clo, chi = oracle.coarse_box(typ, order, it, flo, fhi)
    shape = box_shape(clo, chi)
    line = poly_line(cent, intp, q, clo[d], chi[d] - clo[d] + 1)
    bshape = [1, 1, 1]
    bshape[2 - d] = len(line)
    crse = np.broadcast_to(line.reshape(bshape), shape).copy()[None]
    want = fine_exact(cent, intp, q, flo[d], n)
    wshape = [1, 1, 1]
    wshape[2 - d] = n
    want = np.broadcast_to(want.reshape(wshape), box_shape(flo, fhi))[None].copy()
    return crse, clo, chi, flo, fhi, want


def test_oracle_polynomial_reproduction(cx):
    for typ, order, it, d, q in reproduction_cases():
        crse, clo, chi, flo, fhi, want = make_reproduction(cx, typ, order, it, d, q)
        for pg in (0, 1):
            fine = np.zeros_like(want)
            cx.prolong(typ, order, it, pg, crse, clo, chi, fine, flo, fhi, flo, fhi, 1)
            assert np.array_equal(fine, want), (typ, order, it, d, q, pg)


def test_oracle_conservation_and_round_trip(cx):
    """Conservative order 1 in CCC is CC CONS 2 in every direction: the mean of
    the 8 children equals the coarse value to roundoff for any data, and the
    cell-average restriction undoes the prolongation."""
    rng = np.random.default_rng(3)
    clo, chi = (-3, -3, -3), (12, 12, 12)
    flo, fhi = (0, 0, 0), (19, 19, 19)
    crse = rng.uniform(-1, 1, (2,) + box_shape(clo, chi))
    fine = np.zeros((2,) + box_shape(flo, fhi))
    cx.prolong("conservative", 1, 7, 0, crse, clo, chi, fine, flo, fhi, flo, fhi, 2)
    back = np.zeros_like(crse)
    cx.restrict(7, fine, flo, fhi, back, clo, chi, (0, 0, 0), (9, 9, 9), 2)
    sub = crse[:, 3:13, 3:13, 3:13]
    got = back[:, 3:13, 3:13, 3:13]
    assert np.max(np.abs(got - sub)) <= 4 * np.finfo(float).eps * np.max(np.abs(sub))
    # vertex-centred prolongation injects at even points: restriction is exact
    clo, chi = (-2, -2, -2), (12, 12, 12)
    crse = rng.uniform(-1, 1, (1,) + box_shape(clo, chi))
    fine = np.zeros((1,) + box_shape(flo, fhi))
    cx.prolong("interpolate", 5, 0, 0, crse, clo, chi, fine, flo, fhi, flo, fhi, 1)
    back = np.zeros_like(crse)
    cx.restrict(0, fine, flo, fhi, back, clo, chi, (0, 0, 0), (9, 9, 9), 1)
    assert np.array_equal(back[:, 2:12, 2:12, 2:12], crse[:, 2:12, 2:12, 2:12])


@pytest.mark.parametrize("it", range(8))
def test_oracle_restriction_semantics(cx, it):
    """average_down family: injection in vertex directions, mean of the two
    children in cell directions (AMReX semantics; parity unpinned)."""
    rng = np.random.default_rng(it)
    flo, fhi = (-2, -2, -2), (9, 9, 9)
    clo, chi = (-1, -1, -1), (4, 4, 4)
    rlo, rhi = (-1, -1, -1), (4, 4, 4)
    fine = rng.standard_normal((2,) + box_shape(flo, fhi))
    crse = np.zeros((2,) + box_shape(clo, chi))
    cx.restrict(it, fine, flo, fhi, crse, clo, chi, rlo, rhi, 2)
    cc = [(it >> (2 - d)) & 1 for d in range(3)]
    for k in range(rlo[2], rhi[2] + 1):
        for j in range(rlo[1], rhi[1] + 1):
            for i in range(rlo[0], rhi[0] + 1):
                s = 0.0
                for kr in range(cc[2] + 1):
                    for jr in range(cc[1] + 1):
                        for ir in range(cc[0] + 1):
                            s += fine[:, 2 * k + kr - flo[2], 2 * j + jr - flo[1],
                                      2 * i + ir - flo[0]]
                want = s / (2 ** sum(cc))
                assert np.array_equal(crse[:, k - clo[2], j - clo[1], i - clo[0]], want)


def test_oracle_adjoint_dot_product(cx):
    rng = np.random.default_rng(11)
    for typ, order, it in [("interpolate", 5, 0), ("conservative", 1, 7), ("natural", 3, 3),
                           ("minmod", 3, 5), ("eno", 3, 7), ("poly-cons3lfb", 3, 6)]:
        c = random_case(rng, cx, typ, order, it, ncomp=2, max_n=9, kind="jumps")
        fine = np.zeros((2,) + box_shape(c["flo"], c["fhi"]))
        cx.prolong(typ, order, it, 0, c["crse"], c["clo"], c["chi"], fine, c["flo"], c["fhi"],
                   c["rlo"], c["rhi"], 2)
        v = rng.standard_normal(fine.shape) * region_mask(c["flo"], c["fhi"], c["rlo"], c["rhi"])
        ub = np.zeros_like(c["crse"])
        cx.prolong_adjoint(typ, order, it, 0, c["crse"], c["clo"], c["chi"], v, c["flo"],
                           c["fhi"], c["rlo"], c["rhi"], 2, ub)
        # P is linear at fixed choices: <P u, v> = <u, P^T v> with u = crse
        lhs = np.sum(fine * v)
        rhs = np.sum(c["crse"] * ub)
        assert abs(lhs - rhs) <= 1e-12 * (abs(lhs) + np.sum(np.abs(fine * v))), (typ, lhs, rhs)
