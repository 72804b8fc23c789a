"""The ghost-zone sync of a fine level as plans, the order CarpetX's
FillPatch_ProlongateGhosts runs it (CarpetX/src/fillpatch.cxx:44-137):

  1. FillBoundary of the fine level (same-level halo exchange);
  2. gather of the coarse patches (ParallelCopy from the coarse level's valid
     boxes);
  3. boundary conditions on the coarse patches;
  4. prolongation of every fine patch from its coarse patch (one level plan);
  5. scatter of the fine patches into the fine FABs (ParallelCopy, the FABs'
     valid boxes grown by the ghosts);
  6. boundary conditions on the fine FABs.

The fine patches of a FAB are its ghost shell minus the valid boxes of the
level's FABs, as disjoint boxes; each coarse patch is CoarseBox of its fine
patch.  `SyncChain` builds the six plans once (per regrid) and executes them
in order on a stream; the executions can be captured in one CUDA graph.
With fused=True the prolongation writes the fine patches into the fine FABs
directly and the scatter goes (five plans).  With direct=True (fused too) a
fine patch whose coarse box lies inside one coarse FAB (ghosts included) is
prolongated from that FAB itself, without a coarse patch; a patch that does
not fit one FAB whole is cut at the refined faces of the coarse valid boxes
(cell-centred directions) when every piece then fits.  The gather and the
coarse boundary conditions remain for the other patches only.  That needs
the coarse level's ghosts synced (its FillBoundary and boundary conditions
done), as CarpetX's level loop has them when it fills a fine level's ghosts
(SyncGroupsByDirI syncs the levels coarse to fine); then the FAB holds the
values the gather and the coarse boundary conditions would give the patch.
FABs are CUDA float64 tensors of shape (ncomp, nz, ny, nx) with inclusive
(lo, hi) boxes and their valid boxes (valid_lo, valid_hi)."""
import torch

import carpetx_b200 as cb


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
            out.append((tuple(rlo), tuple(rhi[:d] + [lo[d] - 1] + rhi[d + 1:])))
        if rhi[d] > hi[d]:
            out.append((tuple(rlo[:d] + [hi[d] + 1] + rlo[d + 1:]), tuple(rhi)))
        rlo[d], rhi[d] = lo[d], hi[d]
    return out


def fine_patches(fabs):
    """[(fab index, (lo, hi))]: every FAB's box minus the valid boxes of all
    FABs of the level, as disjoint boxes.  fabs: (lo, hi, valid_lo,
    valid_hi) per FAB."""
    out = []
    for i, (lo, hi, vlo, vhi) in enumerate(fabs):
        parts = subtract((lo, hi), (vlo, vhi))
        for j, other in enumerate(fabs):
            if j != i:
                parts = [q for p in parts for q in subtract(p, (other[2], other[3]))]
        out += [(i, p) for p in parts]
    return out


def split_at(box, cuts):
    """Box as disjoint pieces cut before each fine index of cuts[d] inside it."""
    pieces = [box]
    for d in range(3):
        out = []
        for lo, hi in pieces:
            xs = [c for c in cuts[d] if lo[d] < c <= hi[d]]
            for a, b in zip([lo[d]] + xs, [x - 1 for x in xs] + [hi[d]]):
                out.append((lo[:d] + (a,) + lo[d + 1:], hi[:d] + (b,) + hi[d + 1:]))
        pieces = out
    return pieces


def direct_sources(op, coarse, patches):
    """The pieces of the fine patches [(fab index, box)] and, per piece, the
    coarse FAB (index into coarse: (lo, hi, valid_lo, valid_hi) boxes) whose
    box holds its coarse box, or None (gathered).  A patch is read from one
    coarse FAB whole if it can be, else cut at the refined faces of the
    coarse valid boxes (cell-centred directions) if every piece then can be,
    else gathered whole."""
    def holder(box):
        lo, hi = op.coarse_box(box[0], box[1])
        for ci, c in enumerate(coarse):
            if all(c[0][d] <= lo[d] and hi[d] <= c[1][d] for d in range(3)):
                return ci
        return None

    cuts = [sorted({2 * c[2][d] for c in coarse} | {2 * (c[3][d] + 1) for c in coarse})
            if (op.indextype >> (2 - d)) & 1 else [] for d in range(3)]
    pieces, src = [], []
    for i, p in patches:
        h = holder(p)
        q, hq = [p], [h]
        if h is None:
            cut = split_at(p, cuts)
            hc = [holder(x) for x in cut]
            if len(cut) > 1 and all(x is not None for x in hc):
                q, hq = cut, hc
        pieces += [(i, x) for x in q]
        src += hq
    return pieces, src


def _shape(lo, hi):
    return tuple(int(hi[d]) - int(lo[d]) + 1 for d in (2, 1, 0))


def _npts(lo, hi):
    n = 1
    for s in _shape(lo, hi):
        n *= s
    return n


class SyncChain:
    """The plans of one fine level's ghost sync.  coarse, fine: lists of
    (tensor, lo, hi, valid_lo, valid_hi); op: the prolongation operator;
    nghost: the fine FABs' ghost widths; coarse_bc, fine_bc: the groups'
    boundary-condition specs (cb.bc_struct) on the two levels.  The patch
    buffers are allocated once here.

    fused=True merges steps 4 and 5: every fine patch lies in its own FAB's
    ghost region, so the prolongation writes it there directly, and the fine
    patch buffers and the scatter go.  The result is the same bit for bit:
    the scatter writes each ghost point not covered by a valid box from a
    patch of the same position, and a prolongated value depends only on its
    position and the coarse patch data, which every patch holds alike."""

    def __init__(self, op, ncomp, coarse, fine, nghost, coarse_bc, fine_bc, fused=False,
                 direct=False):
        dev = fine[0][0].device
        fused = fused or direct
        self.fused, self.direct = fused, direct
        self.patches = fine_patches([f[1:] for f in fine])
        self.src = [None] * len(self.patches)
        if direct:
            self.patches, self.src = direct_sources(op, [c[1:] for c in coarse], self.patches)
        self.cpb = [op.coarse_box(p[0], p[1]) for _, p in self.patches]
        self.cp = [None if self.src[k] is not None else
                   torch.full((ncomp,) + _shape(lo, hi), float("nan"), dtype=torch.float64,
                              device=dev) for k, (lo, hi) in enumerate(self.cpb)]
        gathered = [k for k in range(len(self.cpb)) if self.src[k] is None]
        cpfabs = [(self.cp[k], self.cpb[k][0], self.cpb[k][1], self.cpb[k][0], self.cpb[k][1])
                  for k in gathered]
        if fused:
            self.fp = []
            self.prolong_boxes = []
            for k, (i, p) in enumerate(self.patches):
                if self.src[k] is None:
                    c, (lo, hi) = self.cp[k], self.cpb[k]
                else:
                    c, lo, hi = coarse[self.src[k]][:3]
                self.prolong_boxes.append(
                    dict(op=op, ncomp=ncomp, crse=c, crse_lo=lo, crse_hi=hi, fine=fine[i][0],
                         fine_lo=fine[i][1], fine_hi=fine[i][2], reg_lo=p[0], reg_hi=p[1]))
        else:
            self.fp = [torch.full((ncomp,) + _shape(p[0], p[1]), float("nan"),
                                  dtype=torch.float64, device=dev) for _, p in self.patches]
            self.prolong_boxes = [
                dict(op=op, ncomp=ncomp, crse=c, crse_lo=lo, crse_hi=hi, fine=f, fine_lo=p[0],
                     fine_hi=p[1], reg_lo=p[0], reg_hi=p[1])
                for c, (lo, hi), f, (_, p) in zip(self.cp, self.cpb, self.fp, self.patches)]
        self.steps = [("fill_boundary", cb.CopyPlan.fill_boundary(fine, ncomp, nghost))]
        if cpfabs:
            self.steps += [
                ("gather", cb.CopyPlan.parallel_copy(cpfabs, coarse, ncomp)),
                ("coarse_bc", cb.BoundaryPlan(coarse_bc, [f[:3] for f in cpfabs])),
            ]
        self.steps.append(("prolong", cb.LevelPlan(self.prolong_boxes)))
        if not fused:
            fpfabs = [(a, p[0], p[1], p[0], p[1]) for a, (_, p) in zip(self.fp, self.patches)]
            self.steps.append(("scatter", cb.CopyPlan.parallel_copy(fine, fpfabs, ncomp,
                                                                     dst_nghost=nghost)))
        self.steps.append(("fine_bc", cb.BoundaryPlan(fine_bc, [(f[0], f[1], f[2])
                                                                for f in fine])))

    def execute(self, stream=None):
        for _, p in self.steps:
            p.execute(stream)

    def stats(self):
        """Per step: algorithmic bytes and launches of one execution."""
        out = {}
        for name, p in self.steps:
            st = p.stats()
            out[name] = {"bytes": st["bytes"], "launches": st.get("launches")}
        return out

    def close(self):
        for _, p in self.steps:
            p.close()


def tiled_fabs(ncells, fab, nghost, origin=(0, 0, 0)):
    """FAB boxes (lo, hi, valid_lo, valid_hi) tiling the cell-centred block
    origin .. origin + ncells - 1 with valid boxes of `fab` cells (ncells a
    multiple of fab per direction), grown by nghost."""
    out = []
    nb = [ncells[d] // fab[d] for d in range(3)]
    for k in range(nb[2]):
        for j in range(nb[1]):
            for i in range(nb[0]):
                t = (i, j, k)
                vlo = tuple(origin[d] + t[d] * fab[d] for d in range(3))
                vhi = tuple(vlo[d] + fab[d] - 1 for d in range(3))
                out.append((tuple(vlo[d] - nghost[d] for d in range(3)),
                            tuple(vhi[d] + nghost[d] for d in range(3)), vlo, vhi))
    return out
