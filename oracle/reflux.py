"""Test infrastructure: numpy restatement of the reflux of a coarse level
from the next finer one (CarpetX/src/schedule.cxx:2632-2713 through AMReX's
FluxRegister: CrseInit(coarse flux, d, -1), FineAdd(fine flux, d, +1),
Reflux(state, scale, geometry)).  AMReX is not in the reference tree: this
follows the FluxRegister's documented semantics with the operation order of
carpetx_b200/csrc/reflux.cu (parity unpinned).  Every operation is a single
IEEE FP64 numpy operation, so results are bit-comparable.

FABs are (array (ncomp, nz, ny, nx), lo, hi, valid_lo, valid_hi)."""
import numpy as np


def _at(f, q):
    a, lo = f[0], f[1]
    return (slice(None), q[2] - lo[2], q[1] - lo[1], q[0] - lo[0])


def _inside_valid(f, q):
    return all(f[3][d] <= q[d] <= f[4][d] for d in range(3))


def reflux(crse, crse_flux, fine_flux, dx, scale=1.0):
    """In place on the coarse state FABs crse.  crse_flux[d]: the coarse flux
    FABs of direction d (one per state FAB); fine_flux[d]: the fine flux
    FABs of direction d, one per fine box (whose cells are fine_flux[0][b]'s
    valid box less its last x face)."""
    vol = (dx[0] * dx[1]) * dx[2]
    nb = len(fine_flux[0])
    boxes = []
    for b in range(nb):
        lo = tuple(fine_flux[0][b][3])
        hi = list(fine_flux[0][b][4])
        hi[0] -= 1
        boxes.append((lo, tuple(hi)))
    for o in range(6):  # x, y, z low, then x, y, z high
        d, high = o % 3, o // 3
        e1, e2 = [e for e in range(3) if e != d]
        sgn_scale = scale if high else -scale
        for b, (blo, bhi) in enumerate(boxes):
            clo = [v >> 1 for v in blo]
            chi = [v >> 1 for v in bhi]
            face = chi[d] + 1 if high else clo[d]
            fface = bhi[d] + 1 if high else blo[d]
            cell_d = face if high else face - 1
            rng = [range(clo[e], chi[e] + 1) for e in range(3)]
            rng[d] = [cell_d]
            for cz in rng[2]:
                for cy in rng[1]:
                    for cx in rng[0]:
                        c = (cx, cy, cz)
                        owner = [f for f in crse if _inside_valid(f, c)]
                        if not owner:
                            continue
                        fq = list(c)
                        fq[d] = face
                        src = [f for f in crse_flux[d] if _inside_valid(f, fq)]
                        r = -src[0][0][_at(src[0], fq)]
                        for o2 in range(2):
                            for o1 in range(2):
                                q = [0, 0, 0]
                                q[d] = fface
                                q[e1] = 2 * c[e1] + o1
                                q[e2] = 2 * c[e2] + o2
                                f = fine_flux[d][b]
                                r = r + f[0][_at(f, q)]
                        u = owner[0]
                        u[0][_at(u, c)] = u[0][_at(u, c)] + (np.float64(sgn_scale) * r) / vol
