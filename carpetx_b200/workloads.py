"""Seeded synthetic inputs with the shapes and value distributions of the
benchmark configurations (there is no dataset: every input is generated)."""
import numpy as np


def box_shape(lo, hi):
    return tuple(int(hi[d]) - int(lo[d]) + 1 for d in (2, 1, 0))


def fourier_fab(rng, ncomp, lo, hi, nmodes=4, kmin=1, kmax=8, noise=1e-3):
    """ncomp components on the inclusive box [lo, hi], each a sum of `nmodes`
    Fourier modes (integer wavenumbers kmin..kmax per axis over the box,
    amplitudes U[-1,1], random phases) plus U[-noise, noise] noise; FP64,
    generated on the host."""
    shape = box_shape(lo, hi)
    n = np.array(shape[::-1], float)
    x = [np.arange(s, dtype=float)[:, None, None] if a == 2 else
         np.arange(s, dtype=float)[None, :, None] if a == 1 else
         np.arange(s, dtype=float)[None, None, :] for a, s in zip((2, 1, 0), shape)]
    out = np.empty((ncomp,) + shape)
    for c in range(ncomp):
        f = np.zeros(shape)
        for _ in range(nmodes):
            k = rng.integers(kmin, kmax + 1, 3)
            a = rng.uniform(-1, 1)
            ph = rng.uniform(0, 2 * np.pi, 3)
            f += a * (np.sin(2 * np.pi * k[0] * x[2] / n[0] + ph[0])
                      * np.sin(2 * np.pi * k[1] * x[1] / n[1] + ph[1])
                      * np.sin(2 * np.pi * k[2] * x[0] / n[2] + ph[2]))
        out[c] = f + rng.uniform(-noise, noise, shape)
    return out


def mixed_level_boxes(seed, nboxes=512, cmin=8, cmax=64, ghosts=3):
    """The mixed 512-box level: per-direction coarse cell counts
    round(exp(U[ln cmin, ln cmax])), centrings uniform over VVV, CCC, VVC, VCC
    (indextype 0, 7, 1, 3).  Returns per box (indextype, crse_lo, crse_hi,
    fine_lo, fine_hi): coarse cells 0..n-1 (plus the closing vertex in vertex
    directions) with `ghosts` ghost points per side, fine region = the whole
    refined box."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(nboxes):
        n = np.round(np.exp(rng.uniform(np.log(cmin), np.log(cmax), 3))).astype(int)
        it = int(rng.choice([0, 7, 1, 3]))
        cc = [(it >> (2 - d)) & 1 for d in range(3)]
        clo = (-ghosts,) * 3
        chi = tuple(int(n[d] - 1 + (1 - cc[d]) + ghosts) for d in range(3))
        flo = (0, 0, 0)
        fhi = tuple(int(2 * n[d] - 1 + (1 - cc[d])) for d in range(3))
        out.append((it, clo, chi, flo, fhi))
    return out
