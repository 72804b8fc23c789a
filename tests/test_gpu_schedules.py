"""The streaming kernels' schedules and z-chunk caps change only the time:
a mixed level (the four centrings of the throughput configuration, small
and large boxes) transferred under every setting is bit-identical to the
oracle."""
import numpy as np
import pytest
import torch

import carpetx_b200 as cb
from helpers import assert_bitwise, box_shape

pytestmark = pytest.mark.gpu


def test_gpu_every_schedule_matches_oracle(dev, cx):
    from carpetx_b200.workloads import mixed_level_boxes
    L = cb.lib()
    rng = np.random.default_rng(41)
    boxes = []
    for it, clo, chi, flo, fhi in mixed_level_boxes(41, nboxes=24, cmin=4, cmax=40):
        typ, order = ("interpolate", 5) if it == 0 else ("hermite", 3)
        u = rng.standard_normal((2,) + box_shape(clo, chi))
        boxes.append(dict(op=cb.Op(typ, order, it), ncomp=2, crse=torch.from_numpy(u).cuda(),
                          crse_lo=clo, crse_hi=chi,
                          fine=torch.empty((2,) + box_shape(flo, fhi), dtype=torch.float64,
                                           device="cuda"),
                          fine_lo=flo, fine_hi=fhi, reg_lo=flo, reg_hi=fhi, u=u))
    want = []
    for b in boxes:
        w = np.zeros(b["fine"].shape)
        cx.prolong(b["op"].type, b["op"].order, b["op"].indextype, 0, b["u"], b["crse_lo"],
                   b["crse_hi"], w, b["fine_lo"], b["fine_hi"], b["fine_lo"], b["fine_hi"], 2)
        want.append(w)
    try:
        for sched, cap in [(0, 128), (1, 128), (0, 32), (1, 16), (-1, 0)]:
            assert L.cx_debug_set_stream_schedule(-1, sched, cap) == cb.CX_OK
            for b in boxes:
                b["fine"].fill_(np.nan)
            plan = cb.LevelPlan([{k: v for k, v in b.items() if k != "u"} for b in boxes])
            plan.execute()
            assert L.cx_check_device() == cb.CX_OK
            plan.close()
            for i, (b, w) in enumerate(zip(boxes, want)):
                assert_bitwise(b["fine"].cpu().numpy(), w, f"schedule {sched} cap {cap} box {i}")
            # one box alone (box mode) under the same setting
            b = boxes[0]
            b["fine"].fill_(np.nan)
            cb.prolong_box(b["op"], b["crse"], b["crse_lo"], b["crse_hi"], b["fine"],
                           b["fine_lo"], b["fine_hi"], b["fine_lo"], b["fine_hi"], 2)
            assert_bitwise(b["fine"].cpu().numpy(), want[0], f"box mode, schedule {sched}")
    finally:
        L.cx_debug_set_stream_schedule(-1, -1, 0)
