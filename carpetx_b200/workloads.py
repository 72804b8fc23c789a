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


# face conditions (symmetry, boundary) that CarpetX accepts on a face
# (boundaries_impl.hxx:71-108), periodic excluded (it pairs both faces)
BC_FACE_CHOICES = [(0, 0), (1, 0), (3, 0), (3, 1), (0, 2), (0, 3), (0, 4), (0, 5), (1, 2),
                   (1, 3), (1, 4), (1, 5)]


def boundary_spec(rng, ncomp, indextype, domain_n, nghost=3, faces=None, periodic=(False,) * 3):
    """A group's outer conditions on a level whose cell-centred domain is
    0..domain_n[d]-1: per face (symmetry, boundary) drawn from
    BC_FACE_CHOICES unless `faces` ([face][dir] pairs) is given, periodic
    directions periodic on both faces; physical box [0.123, 0.123 + n dx]
    with dx = 0.0371 (no grid point at the origin); per component Dirichlet
    values, Robin values at infinity and reflection parities drawn at
    random."""
    sym = [[0] * 3 for _ in range(2)]
    bc = [[0] * 3 for _ in range(2)]
    for f in range(2):
        for d in range(3):
            s, b = faces[f][d] if faces is not None else \
                BC_FACE_CHOICES[rng.integers(len(BC_FACE_CHOICES))]
            if periodic[d]:
                s, b = 2, 0
            sym[f][d], bc[f][d] = int(s), int(b)
    dx = 0.0371
    return {
        "symmetry": sym, "boundary": bc,
        "domain_lo": (0, 0, 0), "domain_hi": tuple(int(n) - 1 for n in domain_n),
        "prob_lo": (0.123,) * 3, "prob_hi": tuple(0.123 + int(n) * dx for n in domain_n),
        "dx": (dx,) * 3, "indextype": tuple(int(v) for v in indextype),
        "nghost": (nghost,) * 3,
        "dirichlet": rng.uniform(-2, 2, ncomp).tolist(),
        "robin": rng.uniform(-1, 1, ncomp).tolist(),
        "parity": rng.choice([-1, 1], (ncomp, 3)).tolist(),
    }


def tiled_level_fabs(domain_n, box_n, indextype, nghost):
    """FABs (lo, hi) of a level whose domain 0..domain_n-1 is tiled by boxes
    of box_n cells per direction, each grown by nghost (vertex-centred
    directions hold the closing vertex too)."""
    out = []
    nb = [int(domain_n[d]) // int(box_n[d]) for d in range(3)]
    for k in range(nb[2]):
        for j in range(nb[1]):
            for i in range(nb[0]):
                t = (i, j, k)
                lo = tuple(t[d] * box_n[d] - nghost for d in range(3))
                hi = tuple((t[d] + 1) * box_n[d] - 1 + (1 - indextype[d]) + nghost
                           for d in range(3))
                out.append((lo, hi))
    return out


# The level of the boundary-condition benchmark: a 256^3-cell domain in 512
# FABs of 32^3 cells with 3 ghosts, 16 cell-centred components, and every
# kind of condition: reflection (x lower), Dirichlet (x upper), linear
# extrapolation (y lower, z upper), Robin (y upper), Neumann (z lower).
BC_LEVEL_FACES = [[(3, 0), (0, 3), (0, 4)], [(0, 2), (0, 5), (0, 3)]]


def shock_level_boxes(nb_dir=4, n=64, ghosts=3):
    """The boxes of the shock level: nb_dir^3 boxes of n^3 coarse cells
    tiling a cube of (nb_dir n)^3 cells, cell centred.  Per box (index,
    crse_lo, crse_hi, fine_lo, fine_hi): the coarse FAB holds `ghosts` ghost
    cells per side, the fine region is the whole refined box."""
    out = []
    for k in range(nb_dir):
        for j in range(nb_dir):
            for i in range(nb_dir):
                t = (i, j, k)
                clo = tuple(t[d] * n - ghosts for d in range(3))
                chi = tuple((t[d] + 1) * n - 1 + ghosts for d in range(3))
                flo = tuple(2 * t[d] * n for d in range(3))
                fhi = tuple(2 * (t[d] + 1) * n - 1 for d in range(3))
                out.append((len(out), clo, chi, flo, fhi))
    return out


def shock_state(seed, ncells):
    """Parameters of the seeded hydro-like state on a cube of `ncells` cells
    per direction (unit cube, cell centres at (i + 1/2) / ncells): a planar
    shock with a random unit normal through a random point near the centre,
    density and pressure 10x larger on the upstream side; a random velocity
    per side; eight Gaussian blobs added to density and pressure; U[-1e-6,
    1e-6] noise on every variable."""
    rng = np.random.default_rng(seed)
    nrm = rng.standard_normal(3)
    nrm /= np.linalg.norm(nrm)
    return {
        "ncells": int(ncells),
        "normal": nrm,
        "offset": float(nrm @ np.full(3, 0.5) + rng.uniform(-0.15, 0.15)),
        "rho": (1.0, 0.1), "p": (1.0, 0.1),  # upstream, downstream: jumps of 10x
        "vel": rng.uniform(-1, 1, (2, 3)),
        "blob_c": rng.uniform(0, 1, (8, 3)),
        "blob_w": rng.uniform(0.02, 0.08, 8),
        "blob_a": rng.uniform(0.05, 0.3, 8),
        "gamma": 1.4,
        "noise_seed": int(rng.integers(2**31)),
    }


def shock_fab(state, lo, hi, box_id=0):
    """The 5 conserved variables (rho, rho vx, rho vy, rho vz, E) of the
    shock state on the inclusive cell box [lo, hi], shape (5, nz, ny, nx),
    FP64 on the host.  Ghost cells get the same smooth-plus-jump function,
    so neighbouring FABs agree where they overlap; the noise is seeded per
    box."""
    shape = box_shape(lo, hi)
    h = 1.0 / state["ncells"]
    ax = [(np.arange(lo[d], hi[d] + 1, dtype=float) + 0.5) * h for d in range(3)]
    z, y, x = np.meshgrid(ax[2], ax[1], ax[0], indexing="ij")
    n = state["normal"]
    up = (n[0] * x + n[1] * y + n[2] * z) < state["offset"]
    rho = np.where(up, state["rho"][0], state["rho"][1])
    p = np.where(up, state["p"][0], state["p"][1])
    blob = np.zeros(shape)
    for c, w, a in zip(state["blob_c"], state["blob_w"], state["blob_a"]):
        blob += a * np.exp(-((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2) / (2 * w * w))
    rho = rho * (1.0 + blob)
    p = p * (1.0 + blob)
    vel = [np.where(up, state["vel"][0][d], state["vel"][1][d]) for d in range(3)]
    e = p / (state["gamma"] - 1) + 0.5 * rho * (vel[0] ** 2 + vel[1] ** 2 + vel[2] ** 2)
    out = np.stack([rho, rho * vel[0], rho * vel[1], rho * vel[2], e])
    rng = np.random.default_rng(state["noise_seed"] + 7919 * int(box_id))
    out += rng.uniform(-1e-6, 1e-6, out.shape)
    return out
