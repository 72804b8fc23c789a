"""GPU tests of the restriction level plan (cx_restrict_plan_*): a mixed
level of the four centrings of the throughput configuration restricted in
one launch per index type, bit-identical to one cx_restrict_box call per box
and to the oracle (cxo_restrict)."""
import numpy as np
import pytest

from helpers import assert_bitwise

pytestmark = pytest.mark.gpu


def _level(dev, nboxes, ncomp, seed):
    import torch
    from carpetx_b200.workloads import mixed_level_boxes
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    out = []
    for it, clo, chi, flo, fhi in mixed_level_boxes(seed, nboxes=nboxes):
        cc = [(it >> (2 - d)) & 1 for d in range(3)]
        # the coarse points whose children lie in the fine box
        rlo = tuple(flo[d] // 2 for d in range(3))
        rhi = tuple((fhi[d] - cc[d]) // 2 for d in range(3))
        shape_f = tuple(fhi[d] - flo[d] + 1 for d in (2, 1, 0))
        shape_c = tuple(chi[d] - clo[d] + 1 for d in (2, 1, 0))
        fine = torch.empty((ncomp,) + shape_f, dtype=torch.float64, device=dev)
        fine.normal_(generator=g)
        crse = torch.full((ncomp,) + shape_c, 7.0, dtype=torch.float64, device=dev)
        out.append(dict(indextype=it, ncomp=ncomp, fine=fine, fine_lo=flo, fine_hi=fhi,
                        crse=crse, crse_lo=clo, crse_hi=chi, reg_lo=rlo, reg_hi=rhi))
    return out


def test_gpu_restrict_plan_matches_box_calls_and_oracle(cx, dev):
    import torch
    import carpetx_b200 as cb
    boxes = _level(dev, 40, 3, 5)
    want = [b["crse"].clone() for b in boxes]
    for b, w in zip(boxes, want):
        cb.restrict_box(b["indextype"], b["fine"], b["fine_lo"], b["fine_hi"], w, b["crse_lo"],
                        b["crse_hi"], b["reg_lo"], b["reg_hi"], b["ncomp"])
    plan = cb.RestrictPlan(boxes)
    st = plan.stats()
    assert st["launches"] == len({b["indextype"] for b in boxes})
    plan.execute()
    plan.execute()
    torch.cuda.synchronize()
    for i, (b, w) in enumerate(zip(boxes, want)):
        got = b["crse"].cpu().numpy()
        assert_bitwise(got, w.cpu().numpy(), f"box {i}")
        if i < 8:
            ref = np.full(got.shape, 7.0)
            cx.restrict(b["indextype"], b["fine"].cpu().numpy(), b["fine_lo"], b["fine_hi"], ref,
                        b["crse_lo"], b["crse_hi"], b["reg_lo"], b["reg_hi"], b["ncomp"])
            assert_bitwise(got, ref, f"box {i} oracle")
    plan.close()


def test_gpu_restrict_plan_rejects(dev):
    import torch
    import carpetx_b200 as cb
    f = torch.zeros((1, 8, 8, 8), dtype=torch.float64, device=dev)
    c = torch.zeros((1, 4, 4, 4), dtype=torch.float64, device=dev)
    box = dict(indextype=7, ncomp=1, fine=f, fine_lo=(0, 0, 0), fine_hi=(7, 7, 7), crse=c,
               crse_lo=(0, 0, 0), crse_hi=(3, 3, 3), reg_lo=(0, 0, 0), reg_hi=(4, 3, 3))
    with pytest.raises(cb.CxError) as e:
        cb.RestrictPlan([box])
    assert e.value.status == cb.CX_EINVAL
    box.update(indextype=9, reg_hi=(3, 3, 3))
    with pytest.raises(cb.CxError) as e:
        cb.RestrictPlan([box])
    assert e.value.status == cb.CX_EUNSUPPORTED


def test_gpu_restrict_groups_plan_selects_like_restrict(cx, dev):
    """Restrict() of one level through cx_restrict_groups_plan_create: groups
    of every kind the reference tells apart (one time level, several, the
    regrid error, restriction disabled); the restricted time levels equal the
    oracle's restriction bit for bit, the others keep their coarse data."""
    import torch
    import carpetx_b200 as cb
    from oracle.oracle import restrict_selection
    specs = [dict(ntimelevels=1, do_restrict=True), dict(ntimelevels=3, do_restrict=True),
             dict(ntimelevels=2, do_restrict=False),
             dict(ntimelevels=1, do_restrict=True, is_regrid_error=True),
             dict(ntimelevels=2, do_restrict=True)]
    groups = []
    for g, sp in enumerate(specs):
        # a group has one centring: the boxes of the first one drawn; every
        # time level has the same boxes with its own data
        lvl = _level(dev, 8, 1 + g % 3, 100 + g)
        it = lvl[0]["indextype"]
        lvl = [b for b in lvl if b["indextype"] == it]
        tls = []
        for tl in range(sp["ntimelevels"]):
            tls.append([dict(b, fine=torch.randn_like(b["fine"]),
                             crse=torch.full_like(b["crse"], 1.0 + tl)) for b in lvl])
        groups.append(dict(sp, indextype=it, ncomp=1 + g % 3, fabs=tls))
    before = [[[b["crse"].clone() for b in t] for t in gr["fabs"]] for gr in groups]
    plan = cb.RestrictPlan.for_groups(groups)
    want_n = restrict_selection(groups)
    assert plan.restricted == want_n
    plan.execute()
    torch.cuda.synchronize()
    for g, gr in enumerate(groups):
        for tl, t in enumerate(gr["fabs"]):
            for i, b in enumerate(t):
                got = b["crse"].cpu().numpy()
                ref = before[g][tl][i].cpu().numpy()
                if tl < want_n[g]:
                    cx.restrict(b["indextype"], b["fine"].cpu().numpy(), b["fine_lo"],
                                b["fine_hi"], ref, b["crse_lo"], b["crse_hi"], b["reg_lo"],
                                b["reg_hi"], b["ncomp"])
                assert_bitwise(got, ref, f"group {g} time level {tl} FAB {i}")
    plan.close()
