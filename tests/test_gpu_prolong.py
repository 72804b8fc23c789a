"""GPU parity tests of the prolongation through the C ABI: bit-identical to the
reference (golden fixtures produced by the reference operators) and to the
oracle on seeded inputs, including the ENO stencil choice and the
linear-fallback decision point by point."""
import hashlib
import os

import numpy as np
import pytest
import torch

import carpetx_b200 as cb
from config1 import config1_case
from helpers import ALL_OPS, assert_bitwise, box_shape, random_case, region_mask
from test_oracle import golden_cases, make_reproduction, reproduction_cases

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def gpu_prolong(c, pg, fill=np.nan, diag=False):
    crse = torch.from_numpy(np.ascontiguousarray(c["crse"])).cuda()
    fine = torch.full((c["ncomp"],) + box_shape(c["flo"], c["fhi"]), fill, dtype=torch.float64,
                      device="cuda")
    shifts = fb = None
    if diag:
        nreg = int(np.prod(box_shape(c["rlo"], c["rhi"])))
        nblk = 1 if pg else c["ncomp"]
        shifts = torch.full((3 * nreg * nblk,), 99, dtype=torch.int8, device="cuda")
        fb = torch.full((nreg * nblk,), 99, dtype=torch.uint8, device="cuda")
    op = cb.Op(c["typ"], c["order"], c["it"])
    cb.prolong_box(op, crse, c["clo"], c["chi"], fine, c["flo"], c["fhi"], c["rlo"], c["rhi"],
                   c["ncomp"], per_group=pg, shifts=shifts, fallback=fb)
    torch.cuda.synchronize()
    out = fine.cpu().numpy()
    if diag:
        return out, shifts.cpu().numpy(), fb.cpu().numpy()
    return out


def test_gpu_matches_reference_golden(dev):
    for c in golden_cases():
        got = gpu_prolong(c, c["pg"])
        m = region_mask(c["flo"], c["fhi"], c["rlo"], c["rhi"])
        assert_bitwise(got[:, m], c["fine"][:, m], f"{c['typ']} o{c['order']} it{c['it']}")
        assert np.all(np.isnan(got[:, ~m])), "points outside the region were written"


@pytest.mark.parametrize("kind", ["normal", "jumps", "ties"])
def test_gpu_matches_oracle_random(dev, cx, kind):
    rng = np.random.default_rng({"normal": 1, "jumps": 2, "ties": 3}[kind])
    for typ, order, it in ALL_OPS:
        for pg in (0, 1):
            c = random_case(rng, cx, typ, order, it, ncomp=int(rng.integers(1, 4)), max_n=14,
                            kind=kind)
            want = np.full((c["ncomp"],) + box_shape(c["flo"], c["fhi"]), np.nan)
            wsh, wfb = cx.prolong(typ, order, it, pg, c["crse"], c["clo"], c["chi"], want,
                                  c["flo"], c["fhi"], c["rlo"], c["rhi"], c["ncomp"],
                                  want_shifts=True)
            got, gsh, gfb = gpu_prolong(c, pg, diag=True)
            what = f"{typ} o{order} it{it} pg{pg}"
            assert_bitwise(got, want, what)
            assert np.array_equal(gsh, wsh), what + ": ENO stencil choice differs"
            assert np.array_equal(gfb, wfb), what + ": fallback decision differs"


def test_gpu_multi_tile_boxes(dev, cx):
    """Boxes spanning many tiles, odd/negative region bounds, ragged edges."""
    rng = np.random.default_rng(5)
    ops = [("interpolate", 5, 0), ("interpolate", 7, 7), ("conservative", 1, 7),
           ("conservative", 0, 5), ("hermite", 3, 1), ("natural", 7, 3), ("ddf", 5, 6),
           ("minmod", 3, 7), ("eno", 3, 7), ("poly-cons3lfb", 5, 2), ("poly-eno3lfb", 3, 4)]
    for typ, order, it in ops:
        for pg in (0, 1):
            flo = tuple(int(v) for v in rng.integers(-40, 10, 3))
            fhi = tuple(flo[d] + int(rng.integers(30, 75)) for d in range(3))
            rlo = tuple(flo[d] + int(rng.integers(0, 3)) for d in range(3))
            rhi = tuple(fhi[d] - int(rng.integers(0, 3)) for d in range(3))
            clo, chi = cx.coarse_box(typ, order, it, rlo, rhi)
            crse = rng.standard_normal((2,) + box_shape(clo, chi))
            c = dict(typ=typ, order=order, it=it, ncomp=2, crse=crse, clo=clo, chi=chi, flo=flo,
                     fhi=fhi, rlo=rlo, rhi=rhi)
            want = np.full((2,) + box_shape(flo, fhi), np.nan)
            cx.prolong(typ, order, it, pg, crse, clo, chi, want, flo, fhi, rlo, rhi, 2)
            assert_bitwise(gpu_prolong(c, pg), want, f"{typ} o{order} it{it} pg{pg}")


def test_gpu_polynomial_reproduction(dev, cx):
    for typ, order, it, d, q in reproduction_cases():
        crse, clo, chi, flo, fhi, want = make_reproduction(cx, typ, order, it, d, q)
        c = dict(typ=typ, order=order, it=it, ncomp=1, crse=crse, clo=clo, chi=chi, flo=flo,
                 fhi=fhi, rlo=flo, rhi=fhi)
        for pg in (0, 1):
            assert np.array_equal(gpu_prolong(c, pg), want), (typ, order, it, d, q, pg)


def test_gpu_config1_matches_reference_checksum(dev):
    c = dict(config1_case(), typ="interpolate", order=3, it=0, ncomp=1)
    c["rlo"], c["rhi"] = c["flo"], c["fhi"]
    got = gpu_prolong(c, 0)
    want = open(os.path.join(HERE, "golden", "config1_sha256.txt")).read().strip()
    assert hashlib.sha256(np.ascontiguousarray(got).tobytes()).hexdigest() == want


def test_gpu_empty_and_degenerate(dev, cx):
    op = cb.Op("interpolate", 3, 0)
    crse = torch.zeros((1, 10, 10, 10), dtype=torch.float64, device="cuda")
    fine = torch.full((1, 8, 8, 8), 7.0, dtype=torch.float64, device="cuda")
    # empty region: nothing written
    cb.prolong_box(op, crse, (-1, -1, -1), (8, 8, 8), fine, (0, 0, 0), (7, 7, 7), (3, 0, 0),
                   (2, 7, 7), 1)
    torch.cuda.synchronize()
    assert torch.all(fine == 7.0)
    # single point region, odd coordinates
    rng = np.random.default_rng(0)
    c = dict(typ="natural", order=5, it=5, ncomp=3, flo=(-3, -3, -3), fhi=(3, 3, 3),
             rlo=(-1, 1, -3), rhi=(-1, 1, -3))
    c["clo"], c["chi"] = cx.coarse_box("natural", 5, 5, c["rlo"], c["rhi"])
    c["crse"] = rng.standard_normal((3,) + box_shape(c["clo"], c["chi"]))
    want = np.full((3, 7, 7, 7), np.nan)
    cx.prolong("natural", 5, 5, 0, c["crse"], c["clo"], c["chi"], want, c["flo"], c["fhi"],
               c["rlo"], c["rhi"], 3)
    assert_bitwise(gpu_prolong(c, 0), want, "single point")


def test_gpu_rejects_bad_arguments(dev):
    op = cb.Op("conservative", 1, 7)
    crse = torch.zeros((1, 6, 6, 6), dtype=torch.float64, device="cuda")
    fine = torch.zeros((1, 8, 8, 8), dtype=torch.float64, device="cuda")
    with pytest.raises(cb.CxError) as e:  # coarse box misses a ghost layer
        cb.prolong_box(op, crse, (0, 0, 0), (5, 5, 5), fine, (0, 0, 0), (7, 7, 7), (0, 0, 0),
                       (7, 7, 7), 1)
    assert e.value.status == cb.CX_EINVAL
    with pytest.raises(cb.CxError):
        cb.prolong_box(op, crse, (-1, -1, -1), (4, 4, 4), fine, (0, 0, 0), (7, 7, 7), (0, 0, 0),
                       (8, 7, 7), 1)
