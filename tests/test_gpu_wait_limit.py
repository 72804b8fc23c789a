"""The give-up path of the adjoint kernels' bounded waits, forced on the GPU
without a fault: cx_debug_set_wait_limit(0) makes every wait for a plane's
bulk copies give up at once.  The kernel then lets
every copy still in flight into its shared memory land (with the default
bound), returns, and cx_check_device reports CX_ETIMEOUT.  With the default
limit restored, the same box transfers cleanly and matches the oracle."""
import numpy as np
import pytest
import torch

import carpetx_b200 as cb
from helpers import assert_bitwise, box_shape

pytestmark = pytest.mark.gpu


def test_gpu_adjoint_wait_give_up_reported_and_recovered(dev, cx):
    L = cb.lib()
    rng = np.random.default_rng(31)
    op = cb.Op("interpolate", 5, 0)
    flo, fhi = (0, 0, 0), (80, 72, 90)
    clo, chi = op.coarse_box(flo, fhi)
    u = rng.standard_normal((2,) + box_shape(clo, chi))
    v = rng.standard_normal((2,) + box_shape(flo, fhi))
    g_u, g_v = torch.from_numpy(u).cuda(), torch.from_numpy(v).cuda()
    out = torch.zeros(u.shape, dtype=torch.float64, device="cuda")
    assert L.cx_check_device() == cb.CX_OK
    status = []
    try:
        assert L.cx_debug_set_wait_limit(0) == cb.CX_OK
        for _ in range(2):
            cb.prolong_adjoint_box(op, g_u, clo, chi, g_v, flo, fhi, flo, fhi, 2, out)
            status.append(L.cx_check_device())
    finally:
        assert L.cx_debug_set_wait_limit(-1) == cb.CX_OK
    assert status == [cb.CX_ETIMEOUT, cb.CX_ETIMEOUT], status
    # the flag was cleared by the read; the context is intact
    assert L.cx_check_device() == cb.CX_OK
    out.fill_(np.nan)
    cb.prolong_adjoint_box(op, g_u, clo, chi, g_v, flo, fhi, flo, fhi, 2, out)
    assert L.cx_check_device() == cb.CX_OK
    want = np.zeros(u.shape)
    cx.prolong_adjoint("interpolate", 5, 0, 0, u, clo, chi, v, flo, fhi, flo, fhi, 2, want)
    got = out.cpu().numpy()
    assert np.allclose(got, want, rtol=1e-12, atol=1e-12 * np.abs(want).max())


def test_gpu_prolong_wait_give_up_reported_and_recovered(dev, cx):
    """The same for the separable prolongation kernels, whose threads wait
    for each coarse plane's bulk copies: with the limit at 0 the first wait
    gives up, the CTA lets the planes already copied ahead land and stops,
    and cx_check_device reports CX_ETIMEOUT; then a box and a level plan
    transfer cleanly, bit-identical to the oracle."""
    L = cb.lib()
    rng = np.random.default_rng(32)
    cases = [(cb.Op("interpolate", 5, 0), (-1, 0, 2), (70, 41, 57)),
             (cb.Op("hermite", 3, 3), (0, -2, 1), (33, 20, 26))]
    data = []
    for op, flo, fhi in cases:
        clo, chi = op.coarse_box(flo, fhi)
        u = rng.standard_normal((3,) + box_shape(clo, chi))
        data.append((op, flo, fhi, clo, chi, u, torch.from_numpy(u).cuda(),
                     torch.zeros((3,) + box_shape(flo, fhi), dtype=torch.float64, device="cuda")))
    plan = cb.LevelPlan([dict(op=op, ncomp=3, crse=g_u, crse_lo=clo, crse_hi=chi, fine=g_f,
                              fine_lo=flo, fine_hi=fhi, reg_lo=flo, reg_hi=fhi)
                         for op, flo, fhi, clo, chi, u, g_u, g_f in data])
    assert L.cx_check_device() == cb.CX_OK
    status = []
    try:
        assert L.cx_debug_set_wait_limit(0) == cb.CX_OK
        op, flo, fhi, clo, chi, u, g_u, g_f = data[0]
        cb.prolong_box(op, g_u, clo, chi, g_f, flo, fhi, flo, fhi, 3)
        status.append(L.cx_check_device())
        plan.execute()
        status.append(L.cx_check_device())
    finally:
        assert L.cx_debug_set_wait_limit(-1) == cb.CX_OK
    assert status == [cb.CX_ETIMEOUT, cb.CX_ETIMEOUT], status
    assert L.cx_check_device() == cb.CX_OK
    for use_plan in (False, True):
        for *_, g_f in data:
            g_f.fill_(np.nan)
        if use_plan:
            plan.execute()
        else:
            for op, flo, fhi, clo, chi, u, g_u, g_f in data:
                cb.prolong_box(op, g_u, clo, chi, g_f, flo, fhi, flo, fhi, 3)
        assert L.cx_check_device() == cb.CX_OK
        for op, flo, fhi, clo, chi, u, g_u, g_f in data:
            want = np.zeros(g_f.shape)
            cx.prolong(op.type, op.order, op.indextype, 0, u, clo, chi, want, flo, fhi, flo, fhi, 3)
            assert_bitwise(g_f.cpu().numpy(), want)
    plan.close()
