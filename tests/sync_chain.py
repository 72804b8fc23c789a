"""The ghost-zone sync of a fine level on one GPU, as CarpetX's
FillPatch_ProlongateGhosts runs it (CarpetX/src/fillpatch.cxx:44-137), in two
implementations that the tests compare:

  1. FillBoundary of the fine level;
  2. gather of the coarse patches (ParallelCopy from the coarse level's valid
     boxes);
  3. boundary conditions on the coarse patches;
  4. prolongation of every fine patch from its coarse patch;
  5. scatter of the fine patches into the fine FABs (ParallelCopy, the FABs'
     valid boxes grown by the ghosts);
  6. boundary conditions on the fine FABs.

`oracle_chain` runs it on the host with the oracles (oracle/regions.py,
cxo_boundary_box, cxo_prolong); `gpu_chain` with the library's plans, one
launch (or one plan) per step.  The fine patches of a FAB are its ghost shell
minus the other fine FABs' valid boxes, as disjoint boxes; each coarse patch
is CoarseBox of its fine patch.

Level: cell centred, coarse domain 16^3 cells in 8 FABs of 8^3 (3 ghosts),
fine domain 32^3, two fine FABs of 16^3 cells at the lower corner (3 ghosts),
so that patches reach outside the domain on three faces.  The outer faces
carry Dirichlet and Neumann conditions: the thin coarse patches outside the
domain hold every source point those read."""
import numpy as np

from oracle import regions

OP = ("conservative", 1, 7)
NCOMP = 2
NG = (3, 3, 3)
FACES = [[(0, 4), (0, 2), (0, 4)], [(0, 2), (0, 4), (0, 2)]]


def subtract(a, b):
    """Box a minus box b as disjoint boxes (inclusive (lo, hi) pairs)."""
    lo = [max(a[0][d], b[0][d]) for d in range(3)]
    hi = [min(a[1][d], b[1][d]) for d in range(3)]
    if any(lo[d] > hi[d] for d in range(3)):
        return [a]
    out = []
    rlo, rhi = list(a[0]), list(a[1])
    for d in range(3):
        if rlo[d] < lo[d]:
            x = (tuple(rlo), tuple(rhi[:d] + [lo[d] - 1] + rhi[d + 1:]))
            out.append(x)
        if rhi[d] > hi[d]:
            x = (tuple(rlo[:d] + [hi[d] + 1] + rlo[d + 1:]), tuple(rhi))
            out.append(x)
        rlo[d], rhi[d] = lo[d], hi[d]
    return out


def shape(lo, hi):
    return tuple(hi[d] - lo[d] + 1 for d in (2, 1, 0))


def level_layout(wide=False):
    """(coarse FAB boxes, fine FAB boxes, fine patches [(fab index, box)],
    coarse patch boxes); FAB boxes as (lo, hi, valid_lo, valid_hi).  wide:
    one fine FAB of 32 x 16 x 16 cells instead of two of 16^3, so that its
    patches span two coarse FABs in x."""
    from region_cases import tiled
    coarse = tiled((16, 16, 16), (8, 8, 8), (1, 1, 1), NG)
    fine = []
    valid = [((0, 0, 0), (31, 15, 15))] if wide else \
        [((0, 0, 0), (15, 15, 15)), ((16, 0, 0), (31, 15, 15))]
    for vlo, vhi in valid:
        fine.append((tuple(v - 3 for v in vlo), tuple(v + 3 for v in vhi), vlo, vhi))
    patches = []
    for i, (lo, hi, vlo, vhi) in enumerate(fine):
        parts = subtract((lo, hi), (vlo, vhi))
        for j, other in enumerate(fine):
            if j != i:
                parts = [q for p in parts for q in subtract(p, (other[2], other[3]))]
        patches += [(i, p) for p in parts]
    return coarse, fine, patches


def coarse_patch_boxes(cx, patches, op=OP):
    return [cx.coarse_box(*op, p[0], p[1]) for _, p in patches]


def specs(seed):
    from carpetx_b200.workloads import boundary_spec
    rng = np.random.default_rng(seed)
    cs = boundary_spec(rng, NCOMP, (1, 1, 1), (16, 16, 16), nghost=3, faces=FACES)
    fs = boundary_spec(rng, NCOMP, (1, 1, 1), (32, 32, 32), nghost=3, faces=FACES)
    fs["dirichlet"], fs["robin"] = cs["dirichlet"], cs["robin"]
    return cs, fs


def initial_data(seed, coarse, fine, linear=False):
    """Coarse and fine FAB arrays: valid points random (or the linear function
    1/8 + x/4 - y/8 + z/2 of the cell centre in coarse-cell units), ghosts NaN."""
    from region_cases import valid_mask
    rng = np.random.default_rng(seed)

    def fill(lo, hi, vlo, vhi, h):
        a = np.full((NCOMP,) + shape(lo, hi), np.nan)
        m = valid_mask(lo, hi, vlo, vhi)
        if linear:
            z, y, x = np.meshgrid(*[(np.arange(lo[d], hi[d] + 1) + 0.5) * h for d in (2, 1, 0)],
                                  indexing="ij")
            f = 0.125 + 0.25 * x - 0.125 * y + 0.5 * z
            for c in range(NCOMP):
                a[c][m] = (f + c)[m]
        else:
            a[:, m] = rng.uniform(-1, 1, (NCOMP, int(m.sum())))
        return a

    ca = [fill(*b, 1.0) for b in coarse]
    fa = [fill(*b, 0.5) for b in fine]
    return ca, fa


def oracle_chain(cx, seed, linear=False, op=OP, wide=False):
    coarse, fine, patches = level_layout(wide)
    cpb = coarse_patch_boxes(cx, patches, op)
    cs, fs = specs(seed)
    ca, fa = initial_data(seed, coarse, fine, linear)
    ffabs = [[a] + list(b) for a, b in zip(fa, fine)]
    regions.fill_boundary(ffabs, NG)
    cfabs = [[a] + list(b) for a, b in zip(ca, coarse)]
    cp = [[np.full((NCOMP,) + shape(lo, hi), np.nan), lo, hi, lo, hi] for lo, hi in cpb]
    regions.parallel_copy(cp, cfabs)
    for f in cp:
        cx.boundary(cs, f[0], f[1], f[2])
    fp = []
    for (i, (plo, phi)), f in zip(patches, cp):
        out = np.full((NCOMP,) + shape(plo, phi), np.nan)
        cx.prolong(*op, 0, f[0], f[1], f[2], out, plo, phi, plo, phi, NCOMP)
        fp.append([out, plo, phi, plo, phi])
    regions.parallel_copy(ffabs, fp, dst_nghost=NG)
    for f in ffabs:
        cx.boundary(fs, f[0], f[1], f[2])
    return [f[0] for f in ffabs]


def gpu_chain(cx, seed, dev, graph=False):
    """The chain with the plans; graph=True executes it once, then captures
    the six executions into one CUDA graph and replays it twice (every
    execution rewrites the same ghosts from the same valid data)."""
    import torch
    import carpetx_b200 as cb
    coarse, fine, patches = level_layout()
    cpb = coarse_patch_boxes(cx, patches)
    cs, fs = specs(seed)
    ca, fa = initial_data(seed, coarse, fine)
    t = lambda a: torch.from_numpy(a).to(dev)  # noqa: E731
    gc = [t(a) for a in ca]
    gf = [t(a) for a in fa]
    gcp = [torch.full((NCOMP,) + shape(lo, hi), float("nan"), dtype=torch.float64, device=dev)
           for lo, hi in cpb]
    gfp = [torch.full((NCOMP,) + shape(p[0], p[1]), float("nan"), dtype=torch.float64,
                      device=dev) for _, p in patches]
    ffabs = [(a,) + tuple(b) for a, b in zip(gf, fine)]
    cfabs = [(a,) + tuple(b) for a, b in zip(gc, coarse)]
    cpfabs = [(a, lo, hi, lo, hi) for a, (lo, hi) in zip(gcp, cpb)]
    fpfabs = [(a, p[0], p[1], p[0], p[1]) for a, (_, p) in zip(gfp, patches)]
    op = cb.Op(*OP)
    plans = [
        cb.CopyPlan.fill_boundary(ffabs, NCOMP, NG),
        cb.CopyPlan.parallel_copy(cpfabs, cfabs, NCOMP),
        cb.BoundaryPlan(cs, [(a, lo, hi) for a, (lo, hi) in zip(gcp, cpb)]),
        cb.LevelPlan([dict(op=op, ncomp=NCOMP, crse=c, crse_lo=lo, crse_hi=hi, fine=f,
                           fine_lo=p[0], fine_hi=p[1], reg_lo=p[0], reg_hi=p[1])
                      for c, (lo, hi), f, (_, p) in zip(gcp, cpb, gfp, patches)]),
        cb.CopyPlan.parallel_copy(ffabs, fpfabs, NCOMP, dst_nghost=NG),
        cb.BoundaryPlan(fs, [(a, b[0], b[1]) for a, b in zip(gf, fine)]),
    ]
    if graph:
        for p in plans:  # a first execution outside the capture, as a user would
            p.execute()
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            for p in plans:
                p.execute()
        g.replay()
        g.replay()
    else:
        for p in plans:
            p.execute()
    torch.cuda.synchronize()
    out = [a.cpu().numpy() for a in gf]
    if graph:
        del g
    for p in plans:
        p.close()
    return out
