"""numpy restatement of the region copies around a prolongation: AMReX's
MultiFab::FillBoundary and MultiFab::ParallelCopy as CarpetX calls them
(CarpetX/src/fillpatch.cxx:34-37, 63-64, 91-93, 122-124).

TEST INFRASTRUCTURE ONLY: the tests check the CUDA copy plans against it.
AMReX's sources are not in the reference tree, so this restates the
documented behaviour ("parity unpinned"): a destination point takes the value
of the first source, in list order and then periodic-image order (shift 0,
then -period, +period per direction, z outermost), whose box contains it.
Where the sources agree (consistent data) the order does not matter.

A FAB is a list [array (ncomp, nz, ny, nx), lo, hi, valid_lo, valid_hi]; the
arrays are modified in place.  Point by point with masks, not by boxes.
"""
import numpy as np


def images(period):
    per = [[0] + ([-p, p] if p else []) for p in period]
    return [(x, y, z) for z in per[2] for y in per[1] for x in per[0]]


def _coords(lo, hi):
    z, y, x = np.meshgrid(*[np.arange(lo[d], hi[d] + 1) for d in (2, 1, 0)], indexing="ij")
    return x, y, z


def _inside(x, y, z, lo, hi):
    return ((x >= lo[0]) & (x <= hi[0]) & (y >= lo[1]) & (y <= hi[1]) & (z >= lo[2]) &
            (z <= hi[2]))


def _fill(dst, target, sources, period, skip=None):
    """Sets dst's points in `target` (mask) from `sources` [(array, lo, box_lo,
    box_hi)] in order, each image in order; skip = index of the source that
    may not serve at shift 0."""
    a, lo, hi = dst[0], dst[1], dst[2]
    x, y, z = _coords(lo, hi)
    todo = target.copy()
    for j, (sa, slo, blo, bhi) in enumerate(sources):
        for s in images(period):
            if skip == j and s == (0, 0, 0):
                continue
            m = todo & _inside(x - s[0], y - s[1], z - s[2], blo, bhi)
            if not m.any():
                continue
            sx, sy, sz = x[m] - s[0] - slo[0], y[m] - s[1] - slo[1], z[m] - s[2] - slo[2]
            a[:, m] = sa[:, sz, sy, sx]
            todo &= ~m


def fill_boundary(fabs, nghost, period=(0, 0, 0)):
    """mf.FillBoundary(nghost, period) on the FABs, in place."""
    srcs = [(f[0].copy(), f[1], f[3], f[4]) for f in fabs]  # sources: the valid values
    for i, f in enumerate(fabs):
        x, y, z = _coords(f[1], f[2])
        glo = [f[3][d] - nghost[d] for d in range(3)]
        ghi = [f[4][d] + nghost[d] for d in range(3)]
        target = _inside(x, y, z, glo, ghi) & ~_inside(x, y, z, f[3], f[4])
        _fill(f, target, srcs, period, skip=i)


def parallel_copy(dst, src, src_nghost=(0, 0, 0), dst_nghost=(0, 0, 0), period=(0, 0, 0)):
    """dst.ParallelCopy(src, src_nghost, dst_nghost, period), in place."""
    srcs = []
    for f in src:
        blo = [max(f[3][d] - src_nghost[d], f[1][d]) for d in range(3)]
        bhi = [min(f[4][d] + src_nghost[d], f[2][d]) for d in range(3)]
        srcs.append((f[0], f[1], blo, bhi))
    for f in dst:
        x, y, z = _coords(f[1], f[2])
        glo = [f[3][d] - dst_nghost[d] for d in range(3)]
        ghi = [f[4][d] + dst_nghost[d] for d in range(3)]
        _fill(f, _inside(x, y, z, glo, ghi), srcs, period)
