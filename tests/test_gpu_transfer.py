"""GPU tests of restriction, the batched level transfer (one persistent launch,
CUDA-graph capture) and the adjoints, through the C ABI."""
import numpy as np
import pytest
import torch

import carpetx_b200 as cb
from helpers import assert_bitwise, box_shape, region_mask

pytestmark = pytest.mark.gpu


def cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("it", range(8))
def test_gpu_restrict_matches_oracle(dev, cx, it):
    rng = np.random.default_rng(100 + it)
    for _ in range(3):
        flo = tuple(int(v) for v in rng.integers(-20, 0, 3))
        fhi = tuple(flo[d] + int(rng.integers(6, 60)) for d in range(3))
        # coarse region: every coarse point whose children lie in the fine box
        cc = [(it >> (2 - d)) & 1 for d in range(3)]
        rlo = tuple(-((-flo[d]) // 2) for d in range(3))
        rhi = tuple((fhi[d] - cc[d]) // 2 for d in range(3))
        clo = tuple(rlo[d] - 1 for d in range(3))
        chi = tuple(rhi[d] + 2 for d in range(3))
        ncomp = int(rng.integers(1, 4))
        fine = rng.standard_normal((ncomp,) + box_shape(flo, fhi))
        want = np.full((ncomp,) + box_shape(clo, chi), np.nan)
        cx.restrict(it, fine, flo, fhi, want, clo, chi, rlo, rhi, ncomp)
        got = torch.full(want.shape, np.nan, dtype=torch.float64, device="cuda")
        cb.restrict_box(it, cuda(fine), flo, fhi, got, clo, chi, rlo, rhi, ncomp)
        torch.cuda.synchronize()
        assert_bitwise(got.cpu().numpy(), want, f"indextype {it}")


def test_gpu_config2_conservation_round_trip(dev, cx):
    """Conservative order-2 cell-centred prolongation (conservative order 1,
    CCC) of a 128^3 box with 3 ghosts, 8 components of random Fourier modes
    plus noise: bit-identical to the oracle, children average to the coarse
    value to roundoff, and restriction undoes prolongation."""
    from carpetx_b200.workloads import fourier_fab
    clo, chi = (-3, -3, -3), (130, 130, 130)
    flo, fhi = (0, 0, 0), (255, 255, 255)
    crse = fourier_fab(np.random.default_rng(2), 8, clo, chi)
    g_crse = cuda(crse)
    g_fine = torch.empty((8,) + box_shape(flo, fhi), dtype=torch.float64, device="cuda")
    op = cb.Op("conservative", 1, 7)
    for pg in (0, 1):
        cb.prolong_box(op, g_crse, clo, chi, g_fine, flo, fhi, flo, fhi, 8, per_group=pg)
        torch.cuda.synchronize()
        if pg == 0:
            want = np.empty((8,) + box_shape(flo, fhi))
            cx.prolong("conservative", 1, 7, 0, crse, clo, chi, want, flo, fhi, flo, fhi, 8)
            assert_bitwise(g_fine.cpu().numpy(), want, "config 2 prolongation")
            del want
        back = torch.empty_like(g_crse)
        cb.restrict_box(7, g_fine, flo, fhi, back, clo, chi, (0, 0, 0), (127, 127, 127), 8)
        torch.cuda.synchronize()
        inner = (slice(None),) + (slice(3, 131),) * 3
        err = (back[inner] - g_crse[inner]).abs().max().item()
        assert err <= 4 * np.finfo(float).eps * g_crse[inner].abs().max().item()


def mixed_level(rng, nboxes, ncomp, cx=None, smin=4, smax=20):
    """Boxes with log-uniform sizes, 3 ghosts, centrings VVV/CCC/VVC/VCC:
    poly order 5 for VVV, hermite order 3 otherwise."""
    boxes = []
    for b in range(nboxes):
        n = np.round(np.exp(rng.uniform(np.log(smin), np.log(smax), 3))).astype(int)
        it = int(rng.choice([0, 7, 1, 3]))
        typ, order = ("interpolate", 5) if it == 0 else ("hermite", 3)
        cc = [(it >> (2 - d)) & 1 for d in range(3)]
        # coarse cells 0..n-1 (+1 vertex in VC directions), fine = 2n (+1)
        flo = (0, 0, 0)
        fhi = tuple(int(2 * n[d] - 1 + (1 - cc[d])) for d in range(3))
        clo = (-3, -3, -3)
        chi = tuple(int(n[d] - 1 + (1 - cc[d]) + 3) for d in range(3))
        crse = rng.standard_normal((ncomp,) + box_shape(clo, chi))
        boxes.append(dict(typ=typ, order=order, it=it, op=cb.Op(typ, order, it), ncomp=ncomp,
                          crse_np=crse, crse_lo=clo, crse_hi=chi, fine_lo=flo, fine_hi=fhi,
                          reg_lo=flo, reg_hi=fhi))
    return boxes


def test_gpu_level_plan_matches_per_box(dev, cx):
    rng = np.random.default_rng(9)
    boxes = mixed_level(rng, 24, 3)
    for b in boxes:
        b["crse"] = cuda(b["crse_np"])
        b["fine"] = torch.full((3,) + box_shape(b["fine_lo"], b["fine_hi"]), np.nan,
                               dtype=torch.float64, device="cuda")
    plan = cb.LevelPlan(boxes)
    st = plan.stats()
    assert st["fine_points"] == sum(3 * np.prod(box_shape(b["fine_lo"], b["fine_hi"]))
                                    for b in boxes)
    plan.execute()
    torch.cuda.synchronize()
    for b in boxes:
        want = np.full((3,) + box_shape(b["fine_lo"], b["fine_hi"]), np.nan)
        cx.prolong(b["typ"], b["order"], b["it"], 0, b["crse_np"], b["crse_lo"], b["crse_hi"],
                   want, b["fine_lo"], b["fine_hi"], b["reg_lo"], b["reg_hi"], 3)
        assert_bitwise(b["fine"].cpu().numpy(), want, f"level box {b['typ']} it{b['it']}")
    # replay under a captured CUDA graph
    for b in boxes:
        b["fine"].fill_(np.nan)
    s = torch.cuda.Stream()
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        plan.execute(stream=s)
    g.replay()
    g.replay()
    torch.cuda.synchronize()
    for b in boxes:
        want = np.full((3,) + box_shape(b["fine_lo"], b["fine_hi"]), np.nan)
        cx.prolong(b["typ"], b["order"], b["it"], 0, b["crse_np"], b["crse_lo"], b["crse_hi"],
                   want, b["fine_lo"], b["fine_hi"], b["reg_lo"], b["reg_hi"], 3)
        assert_bitwise(b["fine"].cpu().numpy(), want, "graph replay")
    plan.close()


def test_gpu_level_plans_pipelined_from_host(dev, cx):
    """The host-resident pattern of the bench's end-to-end leg: a level split
    into batches of boxes, one plan each, with copy in, transfer and copy out
    on three streams over two steps (the second step's copies in overwrite
    buffers the first step's transfers read).  Also: a plan's launch count is
    one per kernel instantiation and CTA size present."""
    rng = np.random.default_rng(12)
    boxes = mixed_level(rng, 18, 2, smin=3, smax=24)
    csz = [b["crse_np"].size for b in boxes]
    fsz = [2 * int(np.prod(box_shape(b["fine_lo"], b["fine_hi"]))) for b in boxes]
    coff, foff = np.concatenate([[0], np.cumsum(csz)]), np.concatenate([[0], np.cumsum(fsz)])
    h_crse = torch.empty(int(coff[-1]), dtype=torch.float64, pin_memory=True)
    h_fine = torch.full((int(foff[-1]),), np.nan, dtype=torch.float64, pin_memory=True)
    crse = torch.empty(int(coff[-1]), dtype=torch.float64, device="cuda")
    fine = torch.full((int(foff[-1]),), np.nan, dtype=torch.float64, device="cuda")
    for b, c0, f0 in zip(boxes, coff, foff):
        h_crse[c0:c0 + b["crse_np"].size] = torch.from_numpy(b["crse_np"].ravel())
        b["crse"] = crse[c0:c0 + b["crse_np"].size].view(b["crse_np"].shape)
        b["fine"] = fine[f0:f0 + 2 * int(np.prod(box_shape(b["fine_lo"], b["fine_hi"])))].view(
            (2,) + box_shape(b["fine_lo"], b["fine_hi"]))
    cuts = [0, 5, 11, 18]
    plans = [cb.LevelPlan(boxes[a:z]) for a, z in zip(cuts[:-1], cuts[1:])]
    for pl, a, z in zip(plans, cuts[:-1], cuts[1:]):
        kinds = {(b["typ"], b["it"]) for b in boxes[a:z]}
        assert 1 <= pl.stats()["launches"] <= 2 * len(kinds)
    s_in, s_x, s_out = torch.cuda.Stream(), torch.cuda.Stream(), torch.cuda.Stream()
    done_x, done_o = [None] * 3, [None] * 3
    torch.cuda.synchronize()
    for step in range(2):
        for k, (a, z) in enumerate(zip(cuts[:-1], cuts[1:])):
            ev_in, ev_x, ev_o = torch.cuda.Event(), torch.cuda.Event(), torch.cuda.Event()
            with torch.cuda.stream(s_in):
                if done_x[k] is not None:
                    s_in.wait_event(done_x[k])
                crse[coff[a]:coff[z]].copy_(h_crse[coff[a]:coff[z]], non_blocking=True)
                ev_in.record(s_in)
            s_x.wait_event(ev_in)
            if done_o[k] is not None:
                s_x.wait_event(done_o[k])
            plans[k].execute(s_x)
            ev_x.record(s_x)
            with torch.cuda.stream(s_out):
                s_out.wait_event(ev_x)
                h_fine[foff[a]:foff[z]].copy_(fine[foff[a]:foff[z]], non_blocking=True)
                ev_o.record(s_out)
            done_x[k], done_o[k] = ev_x, ev_o
    torch.cuda.synchronize()
    for b, f0 in zip(boxes, foff):
        n = 2 * int(np.prod(box_shape(b["fine_lo"], b["fine_hi"])))
        want = np.full((2,) + box_shape(b["fine_lo"], b["fine_hi"]), np.nan)
        cx.prolong(b["typ"], b["order"], b["it"], 0, b["crse_np"], b["crse_lo"], b["crse_hi"],
                   want, b["fine_lo"], b["fine_hi"], b["reg_lo"], b["reg_hi"], 2)
        assert_bitwise(h_fine[f0:f0 + n].numpy().reshape(want.shape), want,
                       f"pipelined {b['typ']} it{b['it']}")
    for pl in plans:
        pl.close()


def test_gpu_level_plan_limited_and_empty(dev, cx):
    """A level mixing separable and limited (ENO, fallback) boxes and an empty
    region."""
    rng = np.random.default_rng(4)
    specs = [("eno", 3, 7), ("interpolate", 3, 0), ("poly-cons3lfb", 3, 7), ("minmod", 1, 7)]
    boxes = []
    for typ, order, it in specs:
        flo, fhi = (-4, -4, -4), (21, 17, 13)
        clo, chi = cx.coarse_box(typ, order, it, flo, fhi)
        crse = rng.standard_normal((2,) + box_shape(clo, chi))
        boxes.append(dict(typ=typ, order=order, it=it, op=cb.Op(typ, order, it), ncomp=2,
                          crse_np=crse, crse=cuda(crse), crse_lo=clo, crse_hi=chi,
                          fine=torch.full((2,) + box_shape(flo, fhi), np.nan, dtype=torch.float64,
                                          device="cuda"),
                          fine_lo=flo, fine_hi=fhi, reg_lo=flo, reg_hi=fhi))
    e = dict(boxes[1], reg_lo=(0, 0, 0), reg_hi=(-1, 5, 5))
    plan = cb.LevelPlan(boxes + [e])
    plan.execute()
    torch.cuda.synchronize()
    for b in boxes:
        want = np.full((2,) + box_shape(b["fine_lo"], b["fine_hi"]), np.nan)
        cx.prolong(b["typ"], b["order"], b["it"], 0, b["crse_np"], b["crse_lo"], b["crse_hi"],
                   want, b["fine_lo"], b["fine_hi"], b["reg_lo"], b["reg_hi"], 2)
        assert_bitwise(b["fine"].cpu().numpy(), want, f"{b['typ']}")
    plan.close()


@pytest.mark.parametrize("typ,order,it", [("interpolate", 5, 0), ("conservative", 1, 7),
                                          ("natural", 3, 3), ("ddf", 7, 6), ("hermite", 5, 1),
                                          ("interpolate", 7, 7), ("conservative", 0, 2)])
def test_gpu_prolong_adjoint(dev, cx, typ, order, it):
    """Dot-product test <P u, v> = <u, P^T v> to 1e-13 relative, and P^T
    against the oracle's transpose."""
    rng = np.random.default_rng(order * 8 + it)
    flo, fhi = (-5, -3, 2), (30, 27, 21)
    rlo, rhi = (-4, -3, 3), (29, 27, 20)
    clo, chi = cx.coarse_box(typ, order, it, rlo, rhi)
    op = cb.Op(typ, order, it)
    u = rng.standard_normal((2,) + box_shape(clo, chi))
    v = rng.standard_normal((2,) + box_shape(flo, fhi)) * region_mask(flo, fhi, rlo, rhi)
    gu, gv = cuda(u), cuda(v)
    Pu = torch.zeros_like(gv)
    cb.prolong_box(op, gu, clo, chi, Pu, flo, fhi, rlo, rhi, 2)
    PTv = torch.full_like(gu, np.nan)
    cb.prolong_adjoint_box(op, gu, clo, chi, gv, flo, fhi, rlo, rhi, 2, PTv)
    torch.cuda.synchronize()
    lhs = torch.sum(Pu * gv).item()
    rhs = torch.sum(gu * PTv).item()
    scale = torch.sum(torch.abs(Pu * gv)).item()
    assert abs(lhs - rhs) <= 1e-13 * scale, (lhs, rhs)
    want = np.zeros_like(u)
    cx.prolong_adjoint(typ, order, it, 0, u, clo, chi, v, flo, fhi, rlo, rhi, 2, want)
    np.testing.assert_allclose(PTv.cpu().numpy(), want, rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("it", [0, 7, 3])
def test_gpu_restrict_adjoint(dev, cx, it):
    rng = np.random.default_rng(it)
    flo, fhi = (0, 0, 0), (23, 21, 19)
    rlo, rhi = (0, 0, 0), (11, 10, 9)
    clo, chi = (-2, -2, -2), (13, 12, 11)
    f = rng.standard_normal((2,) + box_shape(flo, fhi))
    g = rng.standard_normal((2,) + box_shape(clo, chi))
    Rf = torch.zeros((2,) + box_shape(clo, chi), dtype=torch.float64, device="cuda")
    cb.restrict_box(it, cuda(f), flo, fhi, Rf, clo, chi, rlo, rhi, 2)
    RTg = torch.full((2,) + box_shape(flo, fhi), np.nan, dtype=torch.float64, device="cuda")
    cb.restrict_adjoint_box(it, cuda(g), clo, chi, RTg, flo, fhi, rlo, rhi, 2)
    torch.cuda.synchronize()
    mask = np.zeros(g.shape, bool)
    mask[:, rlo[2] - clo[2]:rhi[2] - clo[2] + 1, rlo[1] - clo[1]:rhi[1] - clo[1] + 1,
         rlo[0] - clo[0]:rhi[0] - clo[0] + 1] = True
    lhs = np.sum(Rf.cpu().numpy() * g * mask)
    rhs = np.sum(f * RTg.cpu().numpy())
    assert abs(lhs - rhs) <= 1e-13 * np.sum(np.abs(f)) * np.max(np.abs(g))
    want = np.zeros_like(f)
    cx.restrict_adjoint(it, g, clo, chi, want, flo, fhi, rlo, rhi, 2)
    np.testing.assert_array_equal(RTg.cpu().numpy(), want)


@pytest.mark.parametrize("typ,order,it", [("interpolate", 5, 0), ("conservative", 1, 7),
                                          ("hermite", 3, 3), ("interpolate", 7, 5),
                                          ("conservative", 0, 2), ("natural", 7, 6)])
def test_gpu_prolong_adjoint_tiled(dev, cx, typ, order, it):
    """P^T on boxes that span several adjoint tiles in x and y and several z
    chunks, with an odd region inside the fine box, against the oracle's
    transpose; every coarse point is overwritten."""
    rng = np.random.default_rng(100 + order * 8 + it)
    flo, fhi = (-7, 3, -2), (196, 150, 29)
    rlo, rhi = (-5, 4, -1), (193, 149, 28)
    clo, chi = cx.coarse_box(typ, order, it, rlo, rhi)
    clo = tuple(c - 1 for c in clo)  # one more coarse layer than the stencils read
    op = cb.Op(typ, order, it)
    u = rng.standard_normal((1,) + box_shape(clo, chi))
    v = rng.standard_normal((1,) + box_shape(flo, fhi))
    PTv = torch.full((1,) + box_shape(clo, chi), np.nan, dtype=torch.float64, device="cuda")
    cb.prolong_adjoint_box(op, cuda(u), clo, chi, cuda(v), flo, fhi, rlo, rhi, 1, PTv)
    torch.cuda.synchronize()
    want = np.zeros_like(u)
    cx.prolong_adjoint(typ, order, it, 0, u, clo, chi, v * region_mask(flo, fhi, rlo, rhi), flo,
                       fhi, rlo, rhi, 1, want)
    got = PTv.cpu().numpy()
    assert not np.any(np.isnan(got)), "coarse points left unwritten"
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-12 * np.max(np.abs(want)))


def test_gpu_adjoint_level_plan(dev, cx):
    """cx_level_plan_create_adjoint: every box's coarse array becomes P^T of
    its fine array, equal bit for bit to cx_prolong_adjoint_box (each coarse
    plane is summed by one work item in fine-plane order, whatever the z
    chunking) and to the oracle's transpose within roundoff; boxes with an
    empty region are zeroed; limited operators are refused."""
    rng = np.random.default_rng(11)
    specs = [("interpolate", 5, 0), ("conservative", 1, 7), ("hermite", 3, 1), ("natural", 5, 6),
             ("interpolate", 3, 7), ("ddf", 5, 3)]
    boxes, per_box = [], []
    for i in range(12):
        typ, order, it = specs[i % len(specs)]
        flo = tuple(int(v) for v in rng.integers(-6, 6, 3))
        fhi = tuple(flo[d] + int(rng.integers(8, 70)) for d in range(3))
        rlo = tuple(flo[d] + int(rng.integers(0, 3)) for d in range(3))
        rhi = tuple(fhi[d] - int(rng.integers(0, 3)) for d in range(3))
        if i == 11:
            rhi = (rlo[0] - 1,) + rhi[1:]  # empty region
        clo, chi = cx.coarse_box(typ, order, it, flo, fhi)
        v = rng.standard_normal((2,) + box_shape(flo, fhi))
        cbar = torch.full((2,) + box_shape(clo, chi), np.nan, dtype=torch.float64, device="cuda")
        boxes.append(dict(op=cb.Op(typ, order, it), typ=typ, order=order, it=it, ncomp=2,
                          crse=cbar, crse_lo=clo, crse_hi=chi, fine=cuda(v), fine_np=v,
                          fine_lo=flo, fine_hi=fhi, reg_lo=rlo, reg_hi=rhi))
    plan = cb.LevelPlan(boxes, adjoint=True)
    plan.execute()
    torch.cuda.synchronize()
    for i, b in enumerate(boxes):
        got = b["crse"].cpu().numpy()
        one = torch.full_like(b["crse"], np.nan)
        cb.prolong_adjoint_box(b["op"], b["crse"], b["crse_lo"], b["crse_hi"], b["fine"],
                               b["fine_lo"], b["fine_hi"], b["reg_lo"], b["reg_hi"], 2, one)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(got, one.cpu().numpy(), err_msg=f"box {i} {b['typ']}")
        want = np.zeros_like(got)
        if i == 11:
            assert np.all(got == 0)
            continue
        mask = region_mask(b["fine_lo"], b["fine_hi"], b["reg_lo"], b["reg_hi"])
        cx.prolong_adjoint(b["typ"], b["order"], b["it"], 0, got, b["crse_lo"], b["crse_hi"],
                           b["fine_np"] * mask, b["fine_lo"], b["fine_hi"], b["reg_lo"],
                           b["reg_hi"], 2, want)
        np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-12 * np.max(np.abs(want)))
    plan.close()
    # no bounded device wait gave up
    assert cb.lib().cx_check_device() == cb.CX_OK, cb.lib().cx_last_error()
    lim = dict(boxes[0], op=cb.Op("minmod", 3, 7))
    lim["crse_lo"], lim["crse_hi"] = cx.coarse_box("minmod", 3, 7, lim["fine_lo"], lim["fine_hi"])
    lim["crse"] = torch.zeros((2,) + box_shape(lim["crse_lo"], lim["crse_hi"]),
                              dtype=torch.float64, device="cuda")
    # a limited operator needs the coarse data it is linearised at
    with pytest.raises(cb.CxError) as e:
        cb.LevelPlan([lim], adjoint=True)
    assert e.value.status == cb.CX_EINVAL


@pytest.mark.parametrize("pg", [0, 1])
def test_gpu_adjoint_level_plan_limited(dev, cx, pg):
    """cx_level_plan_create_adjoint_at: a level mixing limited operators (ENO,
    minmod, active linear fallback, linearised at each box's coarse input)
    with linear ones; every box's coarse array equals cx_prolong_adjoint_box
    bit for bit and the oracle's transpose within roundoff, over two
    executions (the plan's decision scratch is reused)."""
    from helpers import random_case
    rng = np.random.default_rng(21 + pg)
    specs = [("eno", 3, 7), ("minmod", 1, 7), ("interpolate", 5, 0), ("poly-cons3lfb", 3, 7),
             ("eno", 5, 1), ("minmod", 3, 3), ("hermite", 3, 3), ("poly-eno3lfb", 5, 6)]
    boxes = []
    for i, (typ, order, it) in enumerate(specs):
        c = random_case(rng, cx, typ, order, it, ncomp=3, max_n=24,
                        kind="jumps" if i % 2 else "normal")
        v = rng.standard_normal((3,) + box_shape(c["flo"], c["fhi"]))
        boxes.append(dict(op=cb.Op(typ, order, it), typ=typ, order=order, it=it, ncomp=3,
                          crse=torch.full(c["crse"].shape, np.nan, dtype=torch.float64,
                                          device="cuda"),
                          crse_at=cuda(c["crse"]), u=c["crse"], crse_lo=c["clo"],
                          crse_hi=c["chi"], fine=cuda(v), fine_np=v, fine_lo=c["flo"],
                          fine_hi=c["fhi"], reg_lo=c["rlo"], reg_hi=c["rhi"]))
    plan = cb.LevelPlan([{k: b[k] for k in ("op", "ncomp", "crse", "crse_at", "crse_lo",
                                            "crse_hi", "fine", "fine_lo", "fine_hi", "reg_lo",
                                            "reg_hi")} for b in boxes], per_group=bool(pg),
                        adjoint=True)
    for _ in range(2):
        plan.execute()
    torch.cuda.synchronize()
    assert cb.lib().cx_check_device() == cb.CX_OK
    for i, b in enumerate(boxes):
        got = b["crse"].cpu().numpy()
        one = torch.full_like(b["crse"], np.nan)
        cb.prolong_adjoint_box(b["op"], b["crse_at"], b["crse_lo"], b["crse_hi"], b["fine"],
                               b["fine_lo"], b["fine_hi"], b["reg_lo"], b["reg_hi"], 3, one,
                               per_group=bool(pg))
        torch.cuda.synchronize()
        np.testing.assert_array_equal(got, one.cpu().numpy(), err_msg=f"box {i} {b['typ']}")
        mask = region_mask(b["fine_lo"], b["fine_hi"], b["reg_lo"], b["reg_hi"])
        want = np.zeros_like(got)
        cx.prolong_adjoint(b["typ"], b["order"], b["it"], pg, b["u"], b["crse_lo"], b["crse_hi"],
                           b["fine_np"] * mask, b["fine_lo"], b["fine_hi"], b["reg_lo"],
                           b["reg_hi"], 3, want)
        scale = max(1.0, np.abs(want).max())
        np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-12 * scale,
                                   err_msg=f"box {i} {b['typ']} o{b['order']} it{b['it']}")
    plan.close()


@pytest.mark.parametrize("typ,order,it", [("eno", 3, 7), ("eno", 5, 1), ("minmod", 1, 7),
                                          ("minmod", 3, 3), ("poly-cons3lfb", 3, 7),
                                          ("poly-eno3lfb", 5, 6), ("poly-cons3lfb", 5, 0)])
@pytest.mark.parametrize("pg", [0, 1])
def test_gpu_prolong_adjoint_limited(dev, cx, typ, order, it, pg):
    """Adjoint of the limited operators, linearised at the coarse input (ENO
    shift, minmod branch, fallback choice recomputed): against the oracle's
    transpose, and the dot-product identity <P(u), v> = <u, P'(u)^T v>, exact
    for these piecewise-linear maps."""
    from helpers import random_case
    rng = np.random.default_rng(order * 100 + it * 10 + pg)
    for kind in ("jumps", "normal"):
        c = random_case(rng, cx, typ, order, it, ncomp=3, max_n=16, kind=kind)
        op = cb.Op(typ, order, it)
        u, v = c["crse"], rng.standard_normal((3,) + box_shape(c["flo"], c["fhi"]))
        v *= region_mask(c["flo"], c["fhi"], c["rlo"], c["rhi"])
        ptv = torch.full(u.shape, np.nan, dtype=torch.float64, device="cuda")
        cb.prolong_adjoint_box(op, cuda(u), c["clo"], c["chi"], cuda(v), c["flo"], c["fhi"],
                               c["rlo"], c["rhi"], 3, ptv, per_group=bool(pg))
        pu = torch.zeros((3,) + box_shape(c["flo"], c["fhi"]), dtype=torch.float64, device="cuda")
        cb.prolong_box(op, cuda(u), c["clo"], c["chi"], pu, c["flo"], c["fhi"], c["rlo"], c["rhi"],
                       3, per_group=bool(pg))
        torch.cuda.synchronize()
        got = ptv.cpu().numpy()
        want = np.zeros_like(u)
        cx.prolong_adjoint(typ, order, it, pg, u, c["clo"], c["chi"], v, c["flo"], c["fhi"],
                           c["rlo"], c["rhi"], 3, want)
        scale = max(1.0, np.abs(want).max())
        np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-12 * scale,
                                   err_msg=f"{typ} o{order} it{it} pg{pg} {kind}")
        lhs = float(np.sum(pu.cpu().numpy() * v))
        rhs = float(np.sum(u * got))
        assert abs(lhs - rhs) <= 1e-12 * np.sum(np.abs(u * got)), (typ, order, it, pg, lhs, rhs)
    assert cb.lib().cx_check_device() == cb.CX_OK
