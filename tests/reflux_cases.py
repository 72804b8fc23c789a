"""A two-level layout for the reflux tests: a cell-centred coarse level of
32 x 32 x 16 cells in four FABs of 16 x 16 x 16 (2 ghosts), and three fine
boxes, two of them touching (their shared faces are interior to the fine
level) and one at the domain's lower x face (no coarse cell outside it)."""
import numpy as np

NCOMP = 3
DX = (0.125, 0.25, 0.5)


def _face(vlo, vhi, d):
    return tuple(vlo), tuple(v + (e == d) for e, v in enumerate(vhi))


def layout():
    coarse = []
    for j in range(2):
        for i in range(2):
            vlo = (16 * i, 16 * j, 0)
            vhi = (16 * i + 15, 16 * j + 15, 15)
            coarse.append((tuple(v - 2 for v in vlo), tuple(v + 2 for v in vhi), vlo, vhi))
    fine = [((8, 8, 4), (23, 19, 13)), ((24, 8, 4), (39, 19, 13)), ((0, 40, 10), (11, 55, 21))]
    return coarse, fine


def data(seed, dyadic=False):
    """Coarse state FABs, coarse flux FABs per direction, fine flux FABs per
    direction, as (array, lo, hi, valid_lo, valid_hi); random values (or
    multiples of 1/8 below 8, whose sums are exact)."""
    rng = np.random.default_rng(seed)
    coarse, fine = layout()

    def arr(lo, hi):
        shape = (NCOMP,) + tuple(hi[d] - lo[d] + 1 for d in (2, 1, 0))
        if dyadic:
            return rng.integers(-64, 64, shape) / 8.0
        return rng.uniform(-1, 1, shape)

    state = [(arr(lo, hi), lo, hi, vlo, vhi) for lo, hi, vlo, vhi in coarse]
    cflux, fflux = [], []
    for d in range(3):
        cl = []
        for lo, hi, vlo, vhi in coarse:
            flo, fhi = _face(lo, hi, d)
            fvlo, fvhi = _face(vlo, vhi, d)
            cl.append((arr(flo, fhi), flo, fhi, fvlo, fvhi))
        cflux.append(cl)
        fl = []
        for blo, bhi in fine:
            glo = tuple(v - 1 for v in blo)
            ghi = tuple(v + 1 for v in bhi)
            flo, fhi = _face(glo, ghi, d)
            fvlo, fvhi = _face(blo, bhi, d)
            fl.append((arr(flo, fhi), flo, fhi, fvlo, fvhi))
        fflux.append(fl)
    # a shared face holds one flux: the neighbours' copies agree (coarse
    # FABs, and the fine boxes that touch)
    for d in range(3):
        for lst in (cflux[d], fflux[d]):
            for a in lst:
                for b in lst:
                    if a is b:
                        continue
                    lo = [max(a[3][e], b[3][e]) for e in range(3)]
                    hi = [min(a[4][e], b[4][e]) for e in range(3)]
                    if any(lo[e] > hi[e] for e in range(3)):
                        continue
                    sa = tuple(slice(lo[e] - a[1][e], hi[e] - a[1][e] + 1) for e in (2, 1, 0))
                    sb = tuple(slice(lo[e] - b[1][e], hi[e] - b[1][e] + 1) for e in (2, 1, 0))
                    b[0][(slice(None),) + sb] = a[0][(slice(None),) + sa]
    return state, cflux, fflux
