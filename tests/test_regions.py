"""CPU tests of the region copies around a prolongation (AMReX FillBoundary
and ParallelCopy as CarpetX calls them, CarpetX/src/fillpatch.cxx): the numpy
restatement (oracle/regions.py) on levels with known answers, and the C ABI's
piece builder (bounds and argument checks, no launch)."""
import ctypes

import numpy as np
import pytest

from region_cases import in_domain, known_value, random_patches, tiled, valid_mask
from oracle import regions


def level(domain_n, box_n, it, ng, period, ncomp, garbage=np.nan):
    """Tiled FABs holding the known values in their valid boxes, `garbage`
    in their ghosts."""
    out = []
    for lo, hi, vlo, vhi in tiled(domain_n, box_n, it, ng):
        a = known_value(ncomp, lo, hi, period)
        a[:, ~valid_mask(lo, hi, vlo, vhi)] = garbage
        out.append([a, lo, hi, vlo, vhi])
    return out


@pytest.mark.parametrize("it", [(1, 1, 1), (0, 0, 0), (1, 0, 1)])
@pytest.mark.parametrize("periodic", [(0, 0, 0), (1, 1, 1), (1, 0, 0)])
def test_fill_boundary_oracle_known_answer(it, periodic):
    """Every ghost point whose index lies in the domain (after wrapping in
    periodic directions) receives that index's value; the others keep
    theirs."""
    dn, bn, ng = (12, 8, 8), (4, 4, 8), (2, 3, 1)
    period = tuple(dn[d] if periodic[d] else 0 for d in range(3))
    fabs = level(dn, bn, it, ng, period, 2)
    dhi = tuple(dn[d] - 1 + (1 - it[d]) for d in range(3))
    regions.fill_boundary(fabs, ng, period)
    for a, lo, hi, vlo, vhi in fabs:
        want = known_value(2, lo, hi, period)
        m = in_domain(lo, hi, (0, 0, 0), dhi, period)
        assert np.array_equal(a[:, m], want[:, m])
        assert np.isnan(a[:, ~m]).all()


@pytest.mark.parametrize("it", [(1, 1, 1), (0, 1, 0)])
def test_parallel_copy_oracle_known_answer(it):
    """Coarse-patch gather: patches (with ghosts) straddling several coarse
    FABs and the periodic seam receive the index's value from the coarse
    valid boxes; points outside the domain stay unset."""
    dn, period = (16, 16, 8), (16, 0, 0)
    src = level(dn, (8, 4, 8), it, (1, 1, 1), period, 3)
    dhi = tuple(dn[d] - 1 + (1 - it[d]) for d in range(3))
    dst = random_patches(np.random.default_rng(4), 6, dn, 3)
    regions.parallel_copy(dst, src, dst_nghost=(1, 1, 1), period=period)
    for a, lo, hi, vlo, vhi in dst:
        want = known_value(3, lo, hi, period)
        m = (in_domain(lo, hi, (0, 0, 0), dhi, period) &
             valid_mask(lo, hi, tuple(v - 1 for v in vlo), tuple(v + 1 for v in vhi)))
        assert np.array_equal(a[:, m], want[:, m])
        assert np.isnan(a[:, ~m]).all()


def test_region_oracle_first_source_wins():
    """Two vertex-centred FABs sharing the face x = 4 with different values:
    FAB 1's ghost x = 3 comes from FAB 0, FAB 0's ghost x = 5 from FAB 1, and
    the shared face, valid in both, is left alone."""
    a0 = np.full((1, 1, 1, 7), 1.0)  # x -1..5, valid 0..4
    a1 = np.full((1, 1, 1, 7), 2.0)  # x 3..9, valid 4..8
    fabs = [[a0, (-1, 0, 0), (5, 0, 0), (0, 0, 0), (4, 0, 0)],
            [a1, (3, 0, 0), (9, 0, 0), (4, 0, 0), (8, 0, 0)]]
    regions.fill_boundary(fabs, (1, 0, 0))
    assert a0[0, 0, 0, 6] == 2.0 and a0[0, 0, 0, 5] == 1.0
    assert a1[0, 0, 0, 0] == 1.0 and a1[0, 0, 0, 1] == 2.0


def plan_status(kind, fabs_a, fabs_b, ncomp, g1, g2, period):
    """Status of plan creation with placeholder data pointers (no launch is
    ever made); the plan is destroyed if it was created."""
    import carpetx_b200 as cb
    L = cb.lib()

    def arr(fs):
        out = (cb.CxFab * max(1, len(fs)))()
        for i, (lo, hi, vlo, vhi) in enumerate(fs):
            out[i] = cb.CxFab(0x10000, cb._i3(lo), cb._i3(hi), cb._i3(vlo), cb._i3(vhi))
        return out

    h = ctypes.c_void_p()
    if kind == "fb":
        st = L.cx_copy_plan_fill_boundary(arr(fabs_a), len(fabs_a), ncomp, cb._i3(g1),
                                          cb._i3(period), ctypes.byref(h))
    else:
        st = L.cx_copy_plan_parallel_copy(arr(fabs_a), len(fabs_a), arr(fabs_b), len(fabs_b),
                                          ncomp, cb._i3(g1), cb._i3(g2), cb._i3(period),
                                          ctypes.byref(h))
    if st == cb.CX_OK:
        L.cx_copy_plan_destroy(h)
    return st, L.cx_last_error().decode()


def test_copy_plan_host_checks_accept_test_cases():
    """The piece builder accepts the GPU tests' levels: every piece lies in
    its destination FAB and, shifted, in its source FAB.  CX_OK on a machine
    with a device, CX_ECUDA or CX_ENOMEM (the piece upload) without one,
    never CX_EINVAL."""
    import carpetx_b200 as cb
    ok = (cb.CX_OK, cb.CX_ECUDA, cb.CX_ENOMEM)
    for it in ((1, 1, 1), (0, 0, 0), (1, 0, 1)):
        for per in ((0, 0, 0), (12, 8, 8), (12, 0, 0)):
            st, msg = plan_status("fb", tiled((12, 8, 8), (4, 4, 8), it, (2, 3, 1)), None, 2,
                                  (2, 3, 1), None, per)
            assert st in ok, msg
    st, msg = plan_status("fb", tiled((256,) * 3, (32,) * 3, (1, 1, 1), (3, 3, 3)), None, 16,
                          (3, 3, 3), None, (0, 0, 0))
    assert st in ok, msg
    src = tiled((16, 16, 8), (8, 4, 8), (1, 1, 1), (1, 1, 1))
    dst = [(f[1], f[2], f[3], f[4]) for f in random_patches(np.random.default_rng(4), 6,
                                                            (16, 16, 8), 1)]
    st, msg = plan_status("pc", dst, src, 3, (0, 0, 0), (1, 1, 1), (16, 0, 0))
    assert st in ok, msg
    st, msg = plan_status("pc", dst, src, 3, (1, 1, 1), (2, 2, 2), (16, 16, 8))
    assert st in ok, msg


def test_copy_plan_rejects():
    import carpetx_b200 as cb
    bad = [((0, 0, 0), (4, 4, 4), (1, 1, 1), (5, 3, 3))]  # valid box leaves the FAB
    assert plan_status("fb", bad, None, 1, (1, 1, 1), None, (0, 0, 0))[0] == cb.CX_EINVAL
    good = [((0, 0, 0), (4, 4, 4), (1, 1, 1), (3, 3, 3))]
    assert plan_status("fb", good, None, 0, (1, 1, 1), None, (0, 0, 0))[0] == cb.CX_EINVAL
    assert plan_status("fb", good, None, 1, (-1, 1, 1), None, (0, 0, 0))[0] == cb.CX_EINVAL
    assert plan_status("fb", good, None, 1, (1, 1, 1), None, (-4, 0, 0))[0] == cb.CX_EINVAL


def test_restrict_plan_rejects_without_device():
    """cx_restrict_plan_create checks every box as cx_restrict_box does,
    before it touches a device: a region outside the coarse box is
    CX_EINVAL, an index type outside 0..7 CX_EUNSUPPORTED, and the failing
    box is named."""
    import carpetx_b200 as cb
    L = cb.lib()

    def box(it, rhi):
        return cb.CxRestrictBox(it, 1, 0x10000, cb._i3((0, 0, 0)), cb._i3((7, 7, 7)), 0x20000,
                                cb._i3((0, 0, 0)), cb._i3((3, 3, 3)), cb._i3((0, 0, 0)),
                                cb._i3(rhi))

    h = ctypes.c_void_p()
    arr = (cb.CxRestrictBox * 2)(box(7, (3, 3, 3)), box(7, (4, 3, 3)))
    assert L.cx_restrict_plan_create(arr, 2, ctypes.byref(h)) == cb.CX_EINVAL
    assert "box 1" in L.cx_last_error().decode()
    arr = (cb.CxRestrictBox * 1)(box(8, (3, 3, 3)))
    assert L.cx_restrict_plan_create(arr, 1, ctypes.byref(h)) == cb.CX_EUNSUPPORTED
