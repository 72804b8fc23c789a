"""Differentiated prolongation (torch.autograd.Function over the CUDA forward
and the hand-written adjoint kernels): order-5 vertex-centred and
conservative order-2 cell-centred prolongation.  Checks: dot-product test
<P u, v> = <u, P^T v> to 1e-13 relative, central finite differences
(eps = 1e-6) on 200 seeded coarse entries of a weighted sum-of-squares loss,
and the adjoint against the transpose of the oracle's forward assembled
column by column on a 12^3 box."""
import numpy as np
import pytest
import torch

import carpetx_b200 as cb
from carpetx_b200.autograd import prolongate, restrict
from carpetx_b200.workloads import fourier_fab
from helpers import box_shape

pytestmark = pytest.mark.gpu

OPS = [("interpolate", 5, 0), ("conservative", 1, 7)]


def level_boxes(rng, op_spec, nboxes=4):
    typ, order, it = op_spec
    out = []
    for _ in range(nboxes):
        n = np.round(np.exp(rng.uniform(np.log(6), np.log(14), 3))).astype(int)
        cc = [(it >> (2 - d)) & 1 for d in range(3)]
        flo = (0, 0, 0)
        fhi = tuple(int(2 * n[d] - 1 + (1 - cc[d])) for d in range(3))
        clo, chi = cb.Op(typ, order, it).coarse_box(flo, fhi)
        out.append((clo, chi, flo, fhi))
    return out


@pytest.mark.parametrize("spec", OPS)
def test_autograd_dot_product_and_fd(dev, spec):
    typ, order, it = spec
    op = cb.Op(typ, order, it)
    rng = np.random.default_rng(order)
    for clo, chi, flo, fhi in level_boxes(rng, spec):
        u = torch.from_numpy(fourier_fab(rng, 4, clo, chi)).cuda().requires_grad_(True)
        w = torch.from_numpy(rng.uniform(0, 1, (4,) + box_shape(flo, fhi))).cuda()
        fine = prolongate(u, op, clo, chi, flo, fhi)
        loss = torch.sum(w * fine * fine)
        (g,) = torch.autograd.grad(loss, u)
        # dot-product test with the adjoint directly
        v = torch.from_numpy(rng.standard_normal(fine.shape)).cuda()
        ptv = torch.empty_like(u)
        cb.prolong_adjoint_box(op, u.detach(), clo, chi, v, flo, fhi, flo, fhi, 4, ptv)
        lhs = torch.sum(fine.detach() * v).item()
        rhs = torch.sum(u.detach() * ptv).item()
        assert abs(lhs - rhs) <= 1e-13 * torch.sum(torch.abs(fine.detach() * v)).item()
        # central differences on seeded coarse entries
        eps = 1e-6
        flat = u.detach().clone().reshape(-1)
        idx = rng.choice(flat.numel(), size=50, replace=False)
        for i in idx:
            up = flat.clone()
            up[i] += eps
            um = flat.clone()
            um[i] -= eps
            lp = torch.sum(w * prolongate(up.view_as(u), op, clo, chi, flo, fhi) ** 2).item()
            lm = torch.sum(w * prolongate(um.view_as(u), op, clo, chi, flo, fhi) ** 2).item()
            fd = (lp - lm) / (2 * eps)
            an = g.reshape(-1)[i].item()
            assert abs(fd - an) <= 1e-5 * max(1.0, abs(an)), (i, fd, an)


@pytest.mark.parametrize("spec", OPS)
def test_adjoint_matches_assembled_transpose(dev, cx, spec):
    """P^T from the GPU adjoint against the transpose of the oracle's forward
    assembled column by column on a 12^3 coarse box."""
    typ, order, it = spec
    op = cb.Op(typ, order, it)
    g = op.required_ghosts()
    cc = [(it >> (2 - d)) & 1 for d in range(3)]
    clo = (0, 0, 0)
    chi = (11, 11, 11)
    # the largest fine region whose stencils stay inside the 12^3 coarse box
    flo = tuple(2 * g[d] for d in range(3))
    fhi = tuple(2 * (11 - g[d]) + (1 if cc[d] else 0) for d in range(3))
    nc = int(np.prod(box_shape(clo, chi)))
    nf = int(np.prod(box_shape(flo, fhi)))
    P = np.zeros((nf, nc))
    e = np.zeros((1,) + box_shape(clo, chi))
    col = np.zeros((1,) + box_shape(flo, fhi))
    for j in range(nc):
        e.reshape(-1)[:] = 0
        e.reshape(-1)[j] = 1
        cx.prolong(typ, order, it, 0, e, clo, chi, col, flo, fhi, flo, fhi, 1)
        P[:, j] = col.reshape(-1)
    rng = np.random.default_rng(1)
    v = rng.standard_normal((1,) + box_shape(flo, fhi))
    u = torch.zeros((1,) + box_shape(clo, chi), dtype=torch.float64, device="cuda")
    ptv = torch.empty_like(u)
    cb.prolong_adjoint_box(op, u, clo, chi, torch.from_numpy(v).cuda(), flo, fhi, flo, fhi, 1, ptv)
    want = P.T @ v.reshape(-1)
    np.testing.assert_allclose(ptv.cpu().numpy().reshape(-1), want, rtol=1e-13, atol=1e-13)


def test_restrict_autograd(dev):
    rng = np.random.default_rng(2)
    flo, fhi = (0, 0, 0), (15, 13, 11)
    clo, chi = (-1, -1, -1), (8, 7, 6)
    rlo, rhi = (0, 0, 0), (7, 6, 5)
    f = torch.from_numpy(rng.standard_normal((2,) + box_shape(flo, fhi))).cuda().requires_grad_()
    c = restrict(f, 7, flo, fhi, clo, chi, rlo, rhi)
    w = torch.from_numpy(rng.standard_normal(c.shape)).cuda()
    (g,) = torch.autograd.grad(torch.sum(w * c), f)
    # d/df of sum w * mean(children) = w(parent) / 8
    wf = w[:, 1:7, 1:8, 1:9].repeat_interleave(2, 1).repeat_interleave(2, 2).repeat_interleave(2, 3)
    assert torch.equal(g, wf / 8)
