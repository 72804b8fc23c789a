"""torch.autograd.Function wrappers: forward = the CUDA prolongation /
restriction, backward = the hand-written adjoint kernels (gather form, no
atomics).  Used for gradient checks of the transfer operators; the product
path is the C ABI itself."""
import torch

import carpetx_b200 as cb


def _shape(lo, hi):
    return cb.box_shape(lo, hi)


class Prolongate(torch.autograd.Function):
    """fine = P(crse) on one box.  crse: (ncomp, nz, ny, nx) CUDA float64 over
    [crse_lo, crse_hi]; returns the fine FAB over [fine_lo, fine_hi], zero
    outside the region [reg_lo, reg_hi]."""

    @staticmethod
    def forward(ctx, crse, op, crse_lo, crse_hi, fine_lo, fine_hi, reg_lo, reg_hi,
                per_group=False):
        crse = crse.contiguous()
        ncomp = crse.shape[0]
        fine = torch.zeros((ncomp,) + _shape(fine_lo, fine_hi), dtype=torch.float64,
                           device=crse.device)
        cb.prolong_box(op, crse, crse_lo, crse_hi, fine, fine_lo, fine_hi, reg_lo, reg_hi, ncomp,
                       per_group=per_group)
        ctx.save_for_backward(crse)
        ctx.args = (op, crse_lo, crse_hi, fine_lo, fine_hi, reg_lo, reg_hi, per_group)
        return fine

    @staticmethod
    def backward(ctx, gfine):
        (crse,) = ctx.saved_tensors
        op, crse_lo, crse_hi, fine_lo, fine_hi, reg_lo, reg_hi, per_group = ctx.args
        gcrse = torch.empty_like(crse)
        cb.prolong_adjoint_box(op, crse, crse_lo, crse_hi, gfine.contiguous(), fine_lo, fine_hi,
                               reg_lo, reg_hi, crse.shape[0], gcrse, per_group=per_group)
        return (gcrse,) + (None,) * 8


class Restrict(torch.autograd.Function):
    """crse = R(fine) over the coarse region [reg_lo, reg_hi] (zero elsewhere
    in the coarse box)."""

    @staticmethod
    def forward(ctx, fine, indextype, fine_lo, fine_hi, crse_lo, crse_hi, reg_lo, reg_hi):
        fine = fine.contiguous()
        ncomp = fine.shape[0]
        crse = torch.zeros((ncomp,) + _shape(crse_lo, crse_hi), dtype=torch.float64,
                           device=fine.device)
        cb.restrict_box(indextype, fine, fine_lo, fine_hi, crse, crse_lo, crse_hi, reg_lo, reg_hi,
                        ncomp)
        ctx.args = (indextype, fine_lo, fine_hi, crse_lo, crse_hi, reg_lo, reg_hi, ncomp)
        return crse

    @staticmethod
    def backward(ctx, gcrse):
        indextype, fine_lo, fine_hi, crse_lo, crse_hi, reg_lo, reg_hi, ncomp = ctx.args
        gfine = torch.empty((ncomp,) + _shape(fine_lo, fine_hi), dtype=torch.float64,
                            device=gcrse.device)
        cb.restrict_adjoint_box(indextype, gcrse.contiguous(), crse_lo, crse_hi, gfine, fine_lo,
                                fine_hi, reg_lo, reg_hi, ncomp)
        return (gfine,) + (None,) * 7


def prolongate(crse, op, crse_lo, crse_hi, fine_lo, fine_hi, reg_lo=None, reg_hi=None,
               per_group=False):
    reg_lo = fine_lo if reg_lo is None else reg_lo
    reg_hi = fine_hi if reg_hi is None else reg_hi
    return Prolongate.apply(crse, op, tuple(crse_lo), tuple(crse_hi), tuple(fine_lo),
                            tuple(fine_hi), tuple(reg_lo), tuple(reg_hi), per_group)


def restrict(fine, indextype, fine_lo, fine_hi, crse_lo, crse_hi, reg_lo, reg_hi):
    return Restrict.apply(fine, indextype, tuple(fine_lo), tuple(fine_hi), tuple(crse_lo),
                          tuple(crse_hi), tuple(reg_lo), tuple(reg_hi))
