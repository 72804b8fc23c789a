"""Tiled levels for the region-copy tests (FillBoundary, ParallelCopy): FABs
(lo, hi, valid_lo, valid_hi) tiling a domain, and values that are a function
of the periodically wrapped global index, so that every correct fill gives a
known answer wherever a source exists."""
import numpy as np


def tiled(domain_n, box_n, indextype, nghost, origin=(0, 0, 0)):
    """FABs of boxes of box_n cells tiling cells origin..origin+domain_n-1;
    vertex-centred directions hold the closing vertex (adjacent valid boxes
    share it)."""
    out = []
    nb = [domain_n[d] // box_n[d] for d in range(3)]
    for k in range(nb[2]):
        for j in range(nb[1]):
            for i in range(nb[0]):
                t = (i, j, k)
                vlo = tuple(origin[d] + t[d] * box_n[d] for d in range(3))
                vhi = tuple(origin[d] + (t[d] + 1) * box_n[d] - 1 + (1 - indextype[d])
                            for d in range(3))
                lo = tuple(vlo[d] - nghost[d] for d in range(3))
                hi = tuple(vhi[d] + nghost[d] for d in range(3))
                out.append((lo, hi, vlo, vhi))
    return out


def known_value(ncomp, lo, hi, period, origin=(0, 0, 0)):
    """(ncomp, nz, ny, nx) values c 1e9 + x' + 1e3 y' + 1e6 z' of the wrapped
    coordinates (x' = (x - origin) mod period where periodic): exact in FP64."""
    z, y, x = np.meshgrid(*[np.arange(lo[d], hi[d] + 1) for d in (2, 1, 0)], indexing="ij")
    w = []
    for q, d in ((x, 0), (y, 1), (z, 2)):
        q = q - origin[d]
        w.append(np.mod(q, period[d]) if period[d] else q)
    base = w[0] + 1e3 * w[1] + 1e6 * w[2]
    return np.stack([base + 1e9 * c for c in range(ncomp)])


def in_domain(lo, hi, domain_lo, domain_hi, period):
    """Mask of the FAB's points whose index lies in the domain's points
    [domain_lo, domain_hi] in every non-periodic direction."""
    z, y, x = np.meshgrid(*[np.arange(lo[d], hi[d] + 1) for d in (2, 1, 0)], indexing="ij")
    m = np.ones(z.shape, bool)
    for q, d in ((x, 0), (y, 1), (z, 2)):
        if period[d]:
            continue
        m &= (q >= domain_lo[d]) & (q <= domain_hi[d])
    return m


def valid_mask(lo, hi, vlo, vhi):
    z, y, x = np.meshgrid(*[np.arange(lo[d], hi[d] + 1) for d in (2, 1, 0)], indexing="ij")
    return ((x >= vlo[0]) & (x <= vhi[0]) & (y >= vlo[1]) & (y <= vhi[1]) & (z >= vlo[2]) &
            (z <= vhi[2]))


def random_patches(rng, n, domain_n, ncomp, ghost=2):
    """n destination FABs (array of NaN, lo, hi, valid_lo, valid_hi) of random
    size and place, some reaching outside the domain."""
    out = []
    for _ in range(n):
        vlo = tuple(int(rng.integers(-3, domain_n[d] - 2)) for d in range(3))
        vhi = tuple(vlo[d] + int(rng.integers(1, 7)) for d in range(3))
        lo = tuple(v - ghost for v in vlo)
        hi = tuple(v + ghost for v in vhi)
        shape = tuple(hi[d] - lo[d] + 1 for d in (2, 1, 0))
        out.append([np.full((ncomp,) + shape, np.nan), lo, hi, vlo, vhi])
    return out
