"""The oracle's reflux (oracle/reflux.py, AMReX FluxRegister semantics,
parity unpinned) on known answers, and the host-side checks of
cx_reflux_plan_create (no device work)."""
import copy
import ctypes

import numpy as np

import carpetx_b200 as cb
import reflux_cases as rc
from oracle.reflux import reflux


def _outside_cells(blo, bhi):
    """coarse cells just outside a fine box, with the sign of their
    correction: (cell, direction, -1 below a low face / +1 above a high)"""
    clo = [v >> 1 for v in blo]
    chi = [v >> 1 for v in bhi]
    out = []
    for d in range(3):
        for high in (0, 1):
            rng = [range(clo[e], chi[e] + 1) for e in range(3)]
            rng[d] = [chi[d] + 1 if high else clo[d] - 1]
            for z in rng[2]:
                for y in rng[1]:
                    for x in rng[0]:
                        out.append(((x, y, z), d, 1 if high else -1))
    return out


def test_matching_fluxes_change_nothing():
    """Where the four fine fluxes of every register face sum to the coarse
    flux (exactly, dyadic values), every correction is zero."""
    st, cf, ff = rc.data(3, dyadic=True)
    coarse, fine = rc.layout()
    for d in range(3):
        for b, (blo, bhi) in enumerate(fine):
            f = ff[d][b]
            for (c, dd, sgn) in _outside_cells(blo, bhi):
                if dd != d:
                    continue
                face = list(c)
                face[d] = c[d] + 1 if sgn < 0 else c[d]
                src = [g for g in cf[d] if all(g[3][e] <= face[e] <= g[4][e] for e in range(3))]
                if not src:
                    continue
                e1, e2 = [e for e in range(3) if e != d]
                tot = 0.0
                for o2 in range(2):
                    for o1 in range(2):
                        q = [0, 0, 0]
                        q[d] = (bhi[d] + 1) if sgn > 0 else blo[d]
                        q[e1] = 2 * c[e1] + o1
                        q[e2] = 2 * c[e2] + o2
                        tot += f[0][:, q[2] - f[1][2], q[1] - f[1][1], q[0] - f[1][0]]
                for g in src:
                    g[0][:, face[2] - g[1][2], face[1] - g[1][1], face[0] - g[1][0]] = tot
    before = [s[0].copy() for s in st]
    reflux(st, cf, ff, rc.DX)
    for a, b in zip(st, before):
        assert np.array_equal(a[0], b)


def test_correction_of_one_face_known_answer():
    """One x-high register face: the coarse cell above it changes by
    (sum of fine fluxes - coarse flux) / vol."""
    st, cf, ff = rc.data(4, dyadic=True)
    coarse, fine = rc.layout()
    ref = copy.deepcopy(st)
    reflux(st, cf, ff, rc.DX)
    vol = (rc.DX[0] * rc.DX[1]) * rc.DX[2]
    blo, bhi = fine[1]  # x cells 24..39 -> coarse 12..19; the cell above is x = 20
    c = (20, 5, 3)
    f = ff[0][1]
    tot = -cf[0][1][0][:, 3 - cf[0][1][1][2], 5 - cf[0][1][1][1], 20 - cf[0][1][1][0]]
    for o2 in range(2):
        for o1 in range(2):
            q = (40, 2 * 5 + o1, 2 * 3 + o2)
            tot = tot + f[0][:, q[2] - f[1][2], q[1] - f[1][1], q[0] - f[1][0]]
    u = ref[1]
    want = u[0][:, 3 - u[1][2], 5 - u[1][1], 20 - u[1][0]] + tot / vol
    got = st[1][0][:, 3 - u[1][2], 5 - u[1][1], 20 - u[1][0]]
    assert np.array_equal(got, want)


def test_untouched_cells():
    """Only coarse cells next to a fine box change; the box at the domain's
    lower x face has no coarse cell below it."""
    st, cf, ff = rc.data(5)
    coarse, fine = rc.layout()
    ref = copy.deepcopy(st)
    reflux(st, cf, ff, rc.DX)
    near = set(c for blo, bhi in fine for c, _, _ in _outside_cells(blo, bhi))
    for a, b in zip(st, ref):
        lo = a[1]
        changed = np.argwhere((a[0] != b[0]).any(axis=0))
        for z, y, x in changed:
            assert (x + lo[0], y + lo[1], z + lo[2]) in near


def _fab(lo, hi, vlo, vhi):
    f = cb.CxFab()
    f.data = 64
    f.lo, f.hi, f.valid_lo, f.valid_hi = cb._i3(lo), cb._i3(hi), cb._i3(vlo), cb._i3(vhi)
    return f


def test_reflux_plan_rejects_bad_layouts():
    L = cb.lib()
    cs = (cb.CxFab * 1)(_fab((-2,) * 3, (17,) * 3, (0,) * 3, (15,) * 3))
    cfl = [(cb.CxFab * 1)(_fab((-2,) * 3, tuple(17 + (e == d) for e in range(3)), (0,) * 3,
                                tuple(15 + (e == d) for e in range(3)))) for d in range(3)]

    def fine(blo, bhi):
        return [(cb.CxFab * 1)(_fab(tuple(v - 1 for v in blo),
                                    tuple(v + 1 + (e == d) for e, v in enumerate(bhi)), blo,
                                    tuple(v + (e == d) for e, v in enumerate(bhi))))
                for d in range(3)]

    def create(ffl, cfl=cfl):
        cp = (ctypes.POINTER(cb.CxFab) * 3)(*[ctypes.cast(a, ctypes.POINTER(cb.CxFab))
                                              for a in cfl])
        fp = (ctypes.POINTER(cb.CxFab) * 3)(*[ctypes.cast(a, ctypes.POINTER(cb.CxFab))
                                              for a in ffl])
        h = ctypes.c_void_p()
        return L.cx_reflux_plan_create(cs, 1, cp, fp, 1, 2, (ctypes.c_double * 3)(1, 1, 1), 1.0,
                                       ctypes.byref(h)), h
    # odd fine lower corner: not coarsenable by 2
    rc_, h = create(fine((3, 4, 4), (10, 11, 11)))
    assert rc_ == cb.CX_EINVAL and b"coarsenable" in L.cx_last_error()
    # a coarse flux FAB whose valid box is not the state's, face centred
    bad = [(cb.CxFab * 1)(_fab((-2,) * 3, (18,) * 3, (0,) * 3, (16,) * 3)) for d in range(3)]
    rc_, h = create(fine((4, 4, 4), (11, 11, 11)), bad)
    assert rc_ == cb.CX_EINVAL and b"face centred" in L.cx_last_error()
