"""The allocation-free level transfer, cx_level_execute_noalloc.

Some callers cannot allocate device memory while they transfer a level:
- a host framework whose own allocator owns all device memory, where a
  cudaMalloc of ours would fail or take memory that allocator counts on;
- callers that have already handed every byte of the GPU to their allocator.

cx_level_plan_create allocates the device work list with cudaMalloc; this
entry point keeps it in one fixed device array of the library instead.  This
file checks, through the C ABI, that two calls in a row give exactly the
values of the existing level plan (cx_level_plan_*), which the other tests
pin to the reference.  It is collected last, and it works alone in a fresh
process or after the other tests.
"""
import ctypes

import numpy as np
import pytest

import carpetx_b200 as cb

I3 = ctypes.c_int * 3


def _fn():
    L = cb.lib()
    f = L.cx_level_execute_noalloc
    f.argtypes = [ctypes.POINTER(cb.CxBox), ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    return f


def test_noalloc_rejects_too_many_boxes():
    arr = (cb.CxBox * 1)()
    assert _fn()(arr, 1025, 0, None) == cb.CX_EINVAL


def _level(rng, torch, specs, ncomp):
    boxes = []
    for typ, order, it, n in specs:
        cc = [(it >> (2 - d)) & 1 for d in range(3)]
        flo = (0, 0, 0)
        fhi = tuple(int(2 * n[d] - 1 + (1 - cc[d])) for d in range(3))
        op = cb.Op(typ, order, it)
        clo, chi = op.coarse_box(flo, fhi)
        crse = rng.standard_normal((ncomp,) + cb.box_shape(clo, chi))
        boxes.append(dict(op=op, ncomp=ncomp, crse=torch.from_numpy(crse).cuda(), crse_lo=clo,
                          crse_hi=chi, fine_lo=flo, fine_hi=fhi, reg_lo=flo, reg_hi=fhi,
                          fine=torch.full((ncomp,) + cb.box_shape(flo, fhi), np.nan,
                                          dtype=torch.float64, device="cuda")))
    return boxes


def _records(boxes):
    arr = (cb.CxBox * len(boxes))()
    for i, b in enumerate(boxes):
        arr[i] = cb.CxBox(b["op"].handle, b["ncomp"], b["crse"].data_ptr(), I3(*b["crse_lo"]),
                          I3(*b["crse_hi"]), b["fine"].data_ptr(), I3(*b["fine_lo"]),
                          I3(*b["fine_hi"]), I3(*b["reg_lo"]), I3(*b["reg_hi"]))
    return arr


@pytest.mark.gpu
def test_noalloc_matches_level_plan_twice(dev):
    import torch
    from helpers import assert_bitwise
    f = _fn()
    rng = np.random.default_rng(77)
    levels = [
        # mixed separable level: interpolate o5 (VVV), hermite o3 (staggered)
        [("interpolate", 5, 0, (9, 14, 7)), ("hermite", 3, 7, (16, 8, 11)),
         ("hermite", 3, 1, (12, 33, 9)), ("hermite", 3, 3, (70, 10, 8)),
         ("natural", 5, 5, (8, 8, 40))],
        # a different level on the second call, including limited operators
        [("eno", 3, 7, (10, 9, 8)), ("conservative", 1, 7, (24, 12, 20)),
         ("poly-cons3lfb", 3, 6, (9, 11, 10)), ("minmod", 1, 7, (13, 7, 9)),
         ("interpolate", 3, 0, (20, 20, 20))],
    ]
    for call, specs in enumerate(levels):
        boxes = _level(rng, torch, specs, ncomp=3)
        s = torch.cuda.current_stream()
        assert f(_records(boxes), len(boxes), 0, ctypes.c_void_p(s.cuda_stream)) == cb.CX_OK, \
            cb.lib().cx_last_error().decode()
        torch.cuda.synchronize()
        got = [b["fine"].cpu().numpy() for b in boxes]
        for b in boxes:
            b["fine"].fill_(np.nan)
        plan = cb.LevelPlan(boxes)
        plan.execute()
        torch.cuda.synchronize()
        for g, b in zip(got, boxes):
            assert_bitwise(g, b["fine"].cpu().numpy(), f"call {call + 1}: {b['op']}")
        plan.close()
