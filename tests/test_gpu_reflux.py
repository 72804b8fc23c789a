"""GPU test of the reflux plan (cx_reflux_plan_*) against the oracle's
restatement of AMReX's FluxRegister (oracle/reflux.py), bit for bit, on the
layout of tests/reflux_cases.py: two touching fine boxes and one at the
domain's face, four coarse FABs, three components; executed twice (the
corrections add up)."""
import copy

import numpy as np
import pytest
import torch

import carpetx_b200 as cb
import reflux_cases as rc
from helpers import assert_bitwise
from oracle.reflux import reflux

pytestmark = pytest.mark.gpu


def test_gpu_reflux_matches_oracle(dev):
    st, cf, ff = rc.data(7)
    want = copy.deepcopy(st)
    reflux(want, cf, ff, rc.DX, scale=1.0)
    reflux(want, cf, ff, rc.DX, scale=1.0)
    t = lambda fabs: [(torch.from_numpy(a).to(dev),) + tuple(f[1:]) for f in fabs for a in [f[0]]]  # noqa: E731
    g_st = t(st)
    plan = cb.RefluxPlan(g_st, [t(cf[d]) for d in range(3)], [t(ff[d]) for d in range(3)],
                         rc.NCOMP, rc.DX)
    stt = plan.stats()
    assert stt["launches"] == 6 and stt["faces"] > 0
    plan.execute()
    plan.execute()
    torch.cuda.synchronize()
    for i, (g, w) in enumerate(zip(g_st, want)):
        assert_bitwise(g[0].cpu().numpy(), w[0], f"coarse FAB {i}")
    plan.close()
