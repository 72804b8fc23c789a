"""Shared test utilities: seeded FAB generators and bitwise comparison."""
import numpy as np

FAMILIES = {
    "interpolate": (1, 3, 5, 7),
    "conservative": (0, 1),
    "ddf": (1, 3, 5, 7),
    "eno": (3, 5),
    "minmod": (1, 3, 5),
    "hermite": (1, 3, 5),
    "natural": (1, 3, 5, 7),
    "poly-cons3lfb": (1, 3, 5),
    "poly-eno3lfb": (1, 3, 5),
}

ALL_OPS = [(t, o, it) for t, os_ in FAMILIES.items() for o in os_ for it in range(8)]


def box_shape(lo, hi):
    return tuple(int(hi[d]) - int(lo[d]) + 1 for d in (2, 1, 0))


def npts(lo, hi):
    return int(np.prod(box_shape(lo, hi)))


def coarse_data(rng, ncomp, shape, kind):
    """Seeded coarse FAB data: 'normal', 'jumps' (smooth + discontinuity, drives
    ENO shifts and fallbacks), 'ties' (quantised: many equal differences)."""
    if kind == "normal":
        return rng.standard_normal((ncomp,) + shape)
    if kind == "ties":
        return np.round(rng.standard_normal((ncomp,) + shape) * 4) / 4
    z, y, x = np.meshgrid(*[np.arange(s, dtype=float) for s in shape], indexing="ij")
    out = []
    for c in range(ncomp):
        a = rng.uniform(0.1, 0.5, 3)
        f = np.sin(a[0] * x + a[1] * y) + a[2] * z
        nrm = rng.standard_normal(3)
        f = f + 2.0 * ((nrm[0] * x + nrm[1] * y + nrm[2] * z) > rng.uniform(-2, 2) + sum(shape) / 3)
        out.append(f + 1e-3 * rng.standard_normal(shape))
    return np.stack(out)


def random_case(rng, oracle, typ, order, it, ncomp=3, max_n=12, kind="normal"):
    """A random interp() call: fine box, region inside it, coarse box covering
    CoarseBox(region) grown by 0 or 1, coarse data."""
    flo = rng.integers(-9, 9, 3)
    n = rng.integers(1, max_n, 3)
    fhi = flo + n - 1
    rlo = np.minimum(flo + rng.integers(0, 2, 3), fhi)
    rhi = np.maximum(rlo, fhi - rng.integers(0, 2, 3))
    clo, chi = oracle.coarse_box(typ, order, it, rlo, rhi)
    clo = tuple(int(v) for v in np.array(clo) - rng.integers(0, 2, 3))
    chi = tuple(int(v) for v in np.array(chi) + rng.integers(0, 2, 3))
    crse = coarse_data(rng, ncomp, box_shape(clo, chi), kind)
    return dict(typ=typ, order=order, it=it, ncomp=ncomp, crse=crse, clo=clo, chi=chi,
                flo=tuple(int(v) for v in flo), fhi=tuple(int(v) for v in fhi),
                rlo=tuple(int(v) for v in rlo), rhi=tuple(int(v) for v in rhi))


def region_mask(flo, fhi, rlo, rhi):
    m = np.zeros(box_shape(flo, fhi), bool)
    sl = tuple(slice(int(rlo[d]) - int(flo[d]), int(rhi[d]) - int(flo[d]) + 1) for d in (2, 1, 0))
    m[sl] = True
    return m


def bits(a):
    """int64 view with -0.0 mapped to +0.0 (the only representation freedom)."""
    a = np.where(a == 0, 0.0, a)
    return np.ascontiguousarray(a).view(np.int64)


def assert_bitwise(got, want, what=""):
    if not np.array_equal(bits(got), bits(want)):
        d = np.abs(got - want)
        bad = np.count_nonzero(bits(got) != bits(want))
        raise AssertionError(f"{what}: {bad} values differ, max |diff| = {np.nanmax(d)}")


def ulp_distance(a, b):
    """Units in the last place between FP64 arrays (signed-magnitude aware)."""
    ia = bits(a).astype(np.int64)
    ib = bits(b).astype(np.int64)
    ia = np.where(ia < 0, np.int64(-0x8000000000000000) - ia, ia)
    ib = np.where(ib < 0, np.int64(-0x8000000000000000) - ib, ib)
    return np.abs(ia - ib)
