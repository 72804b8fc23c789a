"""Coarse-patch gather for a distributed level transfer (one process per GPU).

Before a fine level is prolongated, every fine box needs the coarse data of
its coarse patch, CoarseBox(fine region), in the memory of the rank that owns
the fine box.  CarpetX obtains it with a parallel copy of the coarse level's
valid regions (no coarse ghosts) into a temporary coarse-patch MultiFab
distributed like the fine patches (CarpetX/src/fillpatch.cxx:86-93,
`mfab_crse_patch.ParallelCopy_nowait(cmfab, ..., IntVect{0}, ...)`), then
interpolates locally (:114-119).  This module is that exchange step:

- every rank computes the same list of pieces (coarse box c owned by rank S)
  x (patch p owned by rank R) = box(c) n patch(p), a pure function of the box
  lists and owner maps, sorted so that both ends of every rank pair post
  their messages in the same order;
- pieces with S == R are copied locally: on CUDA tensors all of them in one
  launch of a copy plan (cx_copy_plan_parallel_copy), elsewhere one tensor
  copy each; the others are packed by S, sent point to point
  (torch.distributed batched isend/irecv: NCCL over NVLink between GPUs,
  gloo between CPU processes) and unpacked by R.

Patch points that no coarse box covers (outside the coarse level) are left as
they are, as ParallelCopy leaves them; boundary conditions fill them.

Boxes are inclusive (lo, hi) index triples; data tensors are shaped
(ncomp, nz, ny, nx) (x fastest, the FArrayBox layout).
"""
from __future__ import annotations

from typing import Dict, List, Optional, Sequence, Tuple

Box = Tuple[Tuple[int, int, int], Tuple[int, int, int]]


def intersect(a: Box, b: Box) -> Optional[Box]:
    lo = tuple(max(a[0][d], b[0][d]) for d in range(3))
    hi = tuple(min(a[1][d], b[1][d]) for d in range(3))
    if any(lo[d] > hi[d] for d in range(3)):
        return None
    return lo, hi


def patch_pieces(coarse_boxes: Sequence[Box], coarse_owner: Sequence[int],
                 patch_boxes: Sequence[Box], patch_owner: Sequence[int]):
    """All pieces (src rank, dst rank, coarse index, patch index, piece box),
    sorted by (src, dst, coarse index, patch index)."""
    out = []
    for pi, pb in enumerate(patch_boxes):
        for ci, cbx in enumerate(coarse_boxes):
            piece = intersect(pb, cbx)
            if piece is not None:
                out.append((int(coarse_owner[ci]), int(patch_owner[pi]), ci, pi, piece))
    out.sort(key=lambda t: t[:4])
    return out


def _view(t, box: Box, piece: Box):
    lo = box[0]
    return t[:, piece[0][2] - lo[2]:piece[1][2] - lo[2] + 1,
             piece[0][1] - lo[1]:piece[1][1] - lo[1] + 1,
             piece[0][0] - lo[0]:piece[1][0] - lo[0] + 1]


class CoarsePatchExchange:
    """The coarse-patch gather of one level pair, for this rank.

    coarse_boxes / coarse_owner: the coarse level's boxes (valid regions) and
    their ranks; patch_boxes / patch_owner: the coarse patches of the fine
    boxes and the ranks of the fine boxes."""

    def __init__(self, coarse_boxes: Sequence[Box], coarse_owner: Sequence[int],
                 patch_boxes: Sequence[Box], patch_owner: Sequence[int], rank: int):
        self.coarse_boxes = [tuple(map(tuple, b)) for b in coarse_boxes]
        self.patch_boxes = [tuple(map(tuple, b)) for b in patch_boxes]
        self.rank = rank
        self.pieces = patch_pieces(self.coarse_boxes, coarse_owner, self.patch_boxes, patch_owner)
        self._plan = None
        self._plan_key = None

    def stats(self) -> Dict[str, int]:
        """Points this rank sends, receives and copies locally (per component)."""
        def npts(b):
            return (b[1][0] - b[0][0] + 1) * (b[1][1] - b[0][1] + 1) * (b[1][2] - b[0][2] + 1)
        s = {"send": 0, "recv": 0, "local": 0}
        for src, dst, _, _, piece in self.pieces:
            if src == self.rank and dst == self.rank:
                s["local"] += npts(piece)
            elif src == self.rank:
                s["send"] += npts(piece)
            elif dst == self.rank:
                s["recv"] += npts(piece)
        return s

    def run(self, coarse_data: Dict[int, "object"], patch_data: Dict[int, "object"]) -> None:
        """Fills this rank's patches (patch index -> tensor) from the coarse
        boxes this rank owns (coarse index -> tensor) and from the other ranks.
        Collective over the default process group when it has more than one
        rank: every rank calls run with its own data."""
        import torch
        import torch.distributed as dist
        ops: List = []
        recvs = []
        local = [(ci, pi, piece) for src, dst, ci, pi, piece in self.pieces
                 if src == self.rank and dst == self.rank]
        plan = self._local_plan(local, coarse_data, patch_data)
        if plan is not None:
            plan.execute()
        for src, dst, ci, pi, piece in self.pieces:
            if src == self.rank and dst == self.rank:
                if plan is None:
                    _view(patch_data[pi], self.patch_boxes[pi], piece).copy_(
                        _view(coarse_data[ci], self.coarse_boxes[ci], piece))
            elif src == self.rank:
                buf = _view(coarse_data[ci], self.coarse_boxes[ci], piece).contiguous()
                ops.append(dist.P2POp(dist.isend, buf, dst))
            elif dst == self.rank:
                ref = patch_data[pi]
                buf = torch.empty(_view(ref, self.patch_boxes[pi], piece).shape, dtype=ref.dtype,
                                  device=ref.device)
                ops.append(dist.P2POp(dist.irecv, buf, src))
                recvs.append((pi, piece, buf))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        for pi, piece, buf in recvs:
            _view(patch_data[pi], self.patch_boxes[pi], piece).copy_(buf)

    def _local_plan(self, local, coarse_data, patch_data):
        """A copy plan for the local pieces when every tensor they involve is
        a CUDA float64 tensor (None otherwise), rebuilt when a tensor
        changes.  The pieces are applied in list order, so where coarse boxes
        overlap (shared vertex faces) the last one sets a point; the plan's
        first source wins, so it gets the coarse boxes in reverse order."""
        if not local:
            return None
        cis = sorted({ci for ci, _, _ in local}, reverse=True)
        pis = sorted({pi for _, pi, _ in local})
        ts = [coarse_data[ci] for ci in cis] + [patch_data[pi] for pi in pis]
        if not all(getattr(t, "is_cuda", False) and str(t.dtype) == "torch.float64"
                   for t in ts):
            return None
        # the caching allocator can hand a freed address to a tensor of
        # another shape, so the key holds each tensor's extents and strides
        # (and with them ncomp) beside its address and device
        key = tuple((t.data_ptr(), t.device.index, tuple(t.shape), tuple(t.stride()))
                    for t in ts)
        if key != self._plan_key:
            from carpetx_b200 import CopyPlan
            ncomp = int(ts[0].shape[0])
            src = [(coarse_data[ci],) + self.coarse_boxes[ci] + self.coarse_boxes[ci]
                   for ci in cis]
            dst = [(patch_data[pi],) + self.patch_boxes[pi] + self.patch_boxes[pi]
                   for pi in pis]
            if self._plan is not None:
                self._plan.close()
            self._plan = CopyPlan.parallel_copy(dst, src, ncomp)
            self._plan_key = key
        return self._plan
