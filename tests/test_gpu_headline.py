"""GPU parity at the benchmark configurations' own sizes, against the oracle.

- The mixed 512-box level of the throughput benchmark (seeded box list of
  carpetx_b200.workloads.mixed_level_boxes: 8-64 coarse cells per direction,
  VVV interpolate o5, VVC/VCC/CCC hermite o3), two components, through a level
  plan replayed from a captured CUDA graph and through the allocation-free
  entry point.  Every fine value is compared bit for bit with the oracle's
  (CarpetX/src/prolongate_3d_rf2_impl.hxx:1256-1689, interp_per_var).  The
  level holds the widest x chunks (129 fine points), whole 128-point z
  columns and boxes on both sides of the 128/256-thread split.
- The shock configuration (carpetx_b200.workloads.shock_state: planar shock
  with a random normal, 10x density and pressure jumps, Gaussian blobs,
  1e-6 noise): two full boxes of 64^3 coarse cells that the shock crosses, 5
  variables, ENO order 3 per variable and per group, values and chosen ENO
  shifts bit for bit (impl.hxx:1415-1517 per variable, :1854-1909 per group),
  so the 8^3 tile seams of the per-coarse-cell kernel see discontinuous
  data; minmod on the same boxes.
"""
import ctypes

import numpy as np
import pytest
import torch

import carpetx_b200 as cb
from carpetx_b200.workloads import mixed_level_boxes, shock_fab, shock_level_boxes, shock_state
from helpers import assert_bitwise, box_shape, npts

pytestmark = pytest.mark.gpu

I3 = ctypes.c_int * 3


def _level512(ncomp, seed=2026):
    rng = np.random.default_rng(seed + 11)
    boxes = []
    for it, clo, chi, flo, fhi in mixed_level_boxes(seed, 512):
        typ, order = ("interpolate", 5) if it == 0 else ("hermite", 3)
        boxes.append(dict(typ=typ, order=order, it=it, op=cb.Op(typ, order, it), ncomp=ncomp,
                          crse_np=rng.standard_normal((ncomp,) + box_shape(clo, chi)),
                          crse_lo=clo, crse_hi=chi, fine_lo=flo, fine_hi=fhi, reg_lo=flo,
                          reg_hi=fhi))
    return boxes


def _units_per_chunk(b):
    """Column units (4 fine y each) per x chunk of the box's streaming tiling
    (x chunks of at most 130 fine points)."""
    w = b["fine_hi"][0] - (b["fine_lo"][0] & ~1) + 1
    if w > 130:
        n = (w + 127) // 128
        w = (w + n - 1) // n
        w += w & 1
    npr = (b["fine_hi"][1] - (b["fine_lo"][1] & ~1)) // 4 + 1
    return npr * w


def _oracle_level(cx, boxes):
    out = []
    for b in boxes:
        want = np.empty((b["ncomp"],) + box_shape(b["fine_lo"], b["fine_hi"]))
        cx.prolong(b["typ"], b["order"], b["it"], 0, b["crse_np"], b["crse_lo"], b["crse_hi"],
                   want, b["fine_lo"], b["fine_hi"], b["reg_lo"], b["reg_hi"], b["ncomp"])
        out.append(want)
    return out


def test_gpu_level512_matches_oracle(dev, cx):
    ncomp = 2
    boxes = _level512(ncomp)
    # the shapes this test is here for
    assert max(b["fine_hi"][0] - b["fine_lo"][0] + 1 for b in boxes) == 129
    assert max(b["fine_hi"][2] - b["fine_lo"][2] + 1 for b in boxes) >= 128
    units = [_units_per_chunk(b) for b in boxes]
    assert min(units) <= 128 < max(units)
    ctot = sum(ncomp * npts(b["crse_lo"], b["crse_hi"]) for b in boxes)
    ftot = sum(ncomp * npts(b["fine_lo"], b["fine_hi"]) for b in boxes)
    crse = torch.empty(ctot, dtype=torch.float64, device="cuda")
    fine = torch.full((ftot,), np.nan, dtype=torch.float64, device="cuda")
    co = fo = 0
    for b in boxes:
        nc, nf = ncomp * npts(b["crse_lo"], b["crse_hi"]), ncomp * npts(b["fine_lo"], b["fine_hi"])
        b["crse"] = crse[co:co + nc].view(b["crse_np"].shape)
        b["crse"].copy_(torch.from_numpy(b["crse_np"]))
        b["fine"] = fine[fo:fo + nf].view((ncomp,) + box_shape(b["fine_lo"], b["fine_hi"]))
        co, fo = co + nc, fo + nf
    want = _oracle_level(cx, boxes)

    def check(what):
        torch.cuda.synchronize()
        host = fine.cpu().numpy()
        fo = 0
        for b, w in zip(boxes, want):
            n = w.size
            assert_bitwise(host[fo:fo + n].reshape(w.shape), w,
                           f"{what}: {b['op']} fine box {b['fine_lo']}..{b['fine_hi']}")
            fo += n

    plan = cb.LevelPlan(boxes)
    s = torch.cuda.Stream()
    plan.execute(stream=s)  # plain execution before the capture
    torch.cuda.synchronize()
    fine.fill_(np.nan)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        plan.execute(stream=s)
    g.replay()
    check("level plan, graph replay")
    del g
    plan.close()

    # the allocation-free entry point on the same level
    arr = (cb.CxBox * len(boxes))()
    for i, b in enumerate(boxes):
        arr[i] = cb.CxBox(b["op"].handle, ncomp, b["crse"].data_ptr(), I3(*b["crse_lo"]),
                          I3(*b["crse_hi"]), b["fine"].data_ptr(), I3(*b["fine_lo"]),
                          I3(*b["fine_hi"]), I3(*b["reg_lo"]), I3(*b["reg_hi"]))
    f = cb.lib().cx_level_execute_noalloc
    f.argtypes = [ctypes.POINTER(cb.CxBox), ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    fine.fill_(np.nan)
    st = torch.cuda.current_stream()
    assert f(arr, len(boxes), 0, ctypes.c_void_p(st.cuda_stream)) == cb.CX_OK, \
        cb.lib().cx_last_error().decode()
    check("allocation-free level transfer")


def _shock_boxes(nbox=2):
    """Two boxes of the shock level that the shock plane crosses (most
    mixed upstream/downstream cells), 5 variables."""
    state = shock_state(4, 256)
    n = state["normal"]
    scored = []
    for bid, clo, chi, flo, fhi in shock_level_boxes():
        c = np.array([(clo[d] + chi[d] + 1) / 2 / 256 for d in range(3)])
        scored.append((abs(n @ c - state["offset"]), bid, clo, chi, flo, fhi))
    scored.sort()
    return state, [s[1:] for s in scored[:nbox]]


@pytest.mark.parametrize("per_group", [0, 1])
def test_gpu_shock_eno_matches_oracle(dev, cx, per_group):
    state, boxes = _shock_boxes()
    op = cb.Op("eno", 3, 7)
    for bid, clo, chi, flo, fhi in boxes:
        crse = shock_fab(state, clo, chi, bid)
        nreg = npts(flo, fhi)
        nblk = 1 if per_group else 5
        want = np.empty((5,) + box_shape(flo, fhi))
        wsh, wfb = cx.prolong("eno", 3, 7, per_group, crse, clo, chi, want, flo, fhi, flo, fhi, 5,
                              want_shifts=True)
        # the shock and its ENO shifts are really there
        assert np.count_nonzero(wsh) > 0.01 * wsh.size
        g_crse = torch.from_numpy(crse).cuda()
        got = torch.full(want.shape, np.nan, dtype=torch.float64, device="cuda")
        gsh = torch.zeros(3 * nreg * nblk, dtype=torch.int8, device="cuda")
        gfb = torch.zeros(nreg * nblk, dtype=torch.uint8, device="cuda")
        cb.prolong_box(op, g_crse, clo, chi, got, flo, fhi, flo, fhi, 5, per_group=per_group,
                       shifts=gsh, fallback=gfb)
        torch.cuda.synchronize()
        assert_bitwise(got.cpu().numpy(), want, f"ENO values, box {bid}")
        assert np.array_equal(gsh.cpu().numpy(), wsh), f"ENO shifts, box {bid}"
        assert np.array_equal(gfb.cpu().numpy(), wfb), f"fallback flags, box {bid}"
        # the same box through a level plan (the level's ENO launches)
        got.fill_(np.nan)
        plan = cb.LevelPlan([dict(op=op, ncomp=5, crse=g_crse, crse_lo=clo, crse_hi=chi,
                                  fine=got, fine_lo=flo, fine_hi=fhi, reg_lo=flo, reg_hi=fhi)],
                            per_group=bool(per_group))
        plan.execute()
        torch.cuda.synchronize()
        plan.close()
        assert_bitwise(got.cpu().numpy(), want, f"ENO level plan, box {bid}")


def test_gpu_shock_minmod_matches_oracle(dev, cx):
    state, boxes = _shock_boxes()
    op = cb.Op("minmod", 1, 7)
    for bid, clo, chi, flo, fhi in boxes:
        crse = shock_fab(state, clo, chi, bid)
        want = np.empty((5,) + box_shape(flo, fhi))
        cx.prolong("minmod", 1, 7, 0, crse, clo, chi, want, flo, fhi, flo, fhi, 5)
        got = torch.full(want.shape, np.nan, dtype=torch.float64, device="cuda")
        plan = cb.LevelPlan([dict(op=op, ncomp=5, crse=torch.from_numpy(crse).cuda(),
                                  crse_lo=clo, crse_hi=chi, fine=got, fine_lo=flo, fine_hi=fhi,
                                  reg_lo=flo, reg_hi=fhi)])
        plan.execute()
        torch.cuda.synchronize()
        plan.close()
        assert_bitwise(got.cpu().numpy(), want, f"minmod, box {bid}")


@pytest.mark.parametrize("typ,order,sub", [("eno", 3, True), ("minmod", 1, False)])
def test_gpu_shock_limited_adjoint_matches_oracle(dev, cx, typ, order, sub):
    """The limited adjoints of the shock configuration at full size: one box
    of 64^3 coarse cells that the shock crosses, through the adjoint level
    plan linearised at the box's coarse data, against the oracle's transpose
    (within roundoff) and the dot-product identity <P(u), v> = <u, P'(u)^T v>.
    Minmod: the whole box, 5 variables.  ENO (whose oracle transpose is
    slow): a 64^3 fine region off the box's corner, across tile seams, 2
    variables."""
    state, boxes = _shock_boxes(1)
    op = cb.Op(typ, order, 7)
    rng = np.random.default_rng(77)
    for bid, clo, chi, flo, fhi in boxes:
        nc = 2 if sub else 5
        crse = np.ascontiguousarray(shock_fab(state, clo, chi, bid)[:nc])
        rlo, rhi = flo, fhi
        if sub:
            rlo = tuple(flo[d] + 37 for d in range(3))
            rhi = tuple(rlo[d] + 63 for d in range(3))
        mask = np.zeros((1,) + box_shape(flo, fhi))
        mask[0, rlo[2] - flo[2]:rhi[2] - flo[2] + 1, rlo[1] - flo[1]:rhi[1] - flo[1] + 1,
             rlo[0] - flo[0]:rhi[0] - flo[0] + 1] = 1.0
        v = rng.standard_normal((nc,) + box_shape(flo, fhi)) * mask
        want = np.zeros_like(crse)
        cx.prolong_adjoint(typ, order, 7, 0, crse, clo, chi, v, flo, fhi, rlo, rhi, nc, want)
        got = torch.full(crse.shape, np.nan, dtype=torch.float64, device="cuda")
        g_crse = torch.from_numpy(crse).cuda()
        plan = cb.LevelPlan([dict(op=op, ncomp=nc, crse=got, crse_at=g_crse, crse_lo=clo,
                                  crse_hi=chi, fine=torch.from_numpy(v).cuda(), fine_lo=flo,
                                  fine_hi=fhi, reg_lo=rlo, reg_hi=rhi)], adjoint=True)
        plan.execute()
        pu = torch.zeros(v.shape, dtype=torch.float64, device="cuda")
        cb.prolong_box(op, g_crse, clo, chi, pu, flo, fhi, rlo, rhi, nc)
        torch.cuda.synchronize()
        plan.close()
        assert cb.lib().cx_check_device() == cb.CX_OK
        g = got.cpu().numpy()
        scale = max(1.0, np.abs(want).max())
        np.testing.assert_allclose(g, want, rtol=1e-12, atol=1e-12 * scale,
                                   err_msg=f"{typ} adjoint, box {bid}")
        lhs = float(np.sum(pu.cpu().numpy() * v))
        rhs = float(np.sum(crse * g))
        assert abs(lhs - rhs) <= 1e-12 * np.sum(np.abs(crse * g)), (typ, lhs, rhs)
