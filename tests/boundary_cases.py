"""Seeded cases for the outer boundary conditions: a group's conditions on a
level (carpetx_b200.workloads.boundary_spec) and one FAB holding data, either
the whole domain grown by the ghosts or a sub-box of it that reaches some of
the domain's faces."""
import numpy as np

from carpetx_b200.workloads import boundary_spec


def fab_data(seed, ncomp, lo, hi):
    """The FAB's input values: U[-1, 1] from the seed, shape (ncomp, nz, ny, nx)."""
    shape = tuple(int(hi[d]) - int(lo[d]) + 1 for d in (2, 1, 0))
    return np.random.default_rng(seed).uniform(-1, 1, (ncomp,) + shape)


def random_bc_case(seed, max_n=7, max_ghost=3, max_comp=3, whole=None):
    """(spec, lo, hi) for case `seed`: domain 2*ghosts+1..max_n cells per
    direction (so that every source point is interior), random centrings,
    conditions (sometimes periodic directions) and components; the FAB is the
    grown domain, or (whole=False, or at random) a sub-box of it that keeps
    at least ghost + 2 interior points per direction."""
    rng = np.random.default_rng(seed)
    g = int(rng.integers(1, max_ghost + 1))
    n = [int(rng.integers(min(2 * g + 2, max_n), max_n + 1)) for _ in range(3)]
    it = tuple(int(v) for v in rng.integers(0, 2, 3))
    per = tuple(bool(v) for v in rng.random(3) < 0.15)
    ncomp = int(rng.integers(1, max_comp + 1))
    spec = boundary_spec(rng, ncomp, it, n, nghost=g, periodic=per)
    lo, hi = [], []
    if whole is None:
        whole = rng.random() < 0.5
    for d in range(3):
        top = n[d] - 1 + (1 - it[d])  # last interior point
        a, b = -g, top + g
        if not whole:
            # keep one side, cut the other inside the interior (if possible)
            keep = int(rng.integers(0, 3))  # 0 lower, 1 upper, 2 both
            span = g + 2
            if keep == 0 and top - span >= 0:
                b = int(rng.integers(span, top + 1))
            elif keep == 1 and top - span >= 0:
                a = int(rng.integers(0, top - span + 1))
        lo.append(a)
        hi.append(b)
    return spec, tuple(lo), tuple(hi)


def outside_mask(spec, lo, hi):
    """True at the FAB's points outside the domain interior."""
    shape = tuple(int(hi[d]) - int(lo[d]) + 1 for d in (2, 1, 0))
    m = np.zeros(shape, bool)
    for d, axis in ((0, 2), (1, 1), (2, 0)):
        imin = spec["domain_lo"][d]
        imax = spec["domain_hi"][d] + 1 + (1 - spec["indextype"][d])
        c = np.arange(lo[d], hi[d] + 1)
        out = (c < imin) | (c >= imax)
        sl = [None, None, None]
        sl[axis] = slice(None)
        m |= out[tuple(sl)]
    return m
