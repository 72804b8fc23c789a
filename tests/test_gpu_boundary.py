"""GPU tests of the outer boundary conditions (cx_boundary_box and the
boundary level plan) against the oracle (cxo_boundary_box, pinned to the
reference's BoundaryCondition) and the reference's golden fixture: bit-exact
on every point of every FAB."""
import numpy as np
import pytest

from boundary_cases import fab_data, outside_mask, random_bc_case
from helpers import assert_bitwise

pytestmark = pytest.mark.gpu


def _dev(a, dev):
    import torch
    return torch.from_numpy(a).to(dev)


def test_gpu_boundary_box_matches_oracle(cx, dev):
    import carpetx_b200 as cb
    for seed in range(2000, 2150):
        spec, lo, hi = random_bc_case(seed, max_n=10, max_ghost=3, max_comp=5)
        a = fab_data(seed, len(spec["dirichlet"]), lo, hi)
        t = _dev(a, dev)
        cb.boundary_box(spec, t, lo, hi)
        cx.boundary(spec, a, lo, hi)
        assert_bitwise(t.cpu().numpy(), a, f"case {seed}")


def test_gpu_boundary_box_matches_golden(dev):
    import carpetx_b200 as cb
    from test_boundary import golden_cases
    for seed, spec, lo, hi, want in golden_cases():
        a = fab_data(seed, len(spec["dirichlet"]), lo, hi)
        t = _dev(a, dev)
        cb.boundary_box(spec, t, lo, hi)
        got = t.cpu().numpy()
        m = outside_mask(spec, lo, hi)
        assert_bitwise(got[:, m], want, f"case {seed}")
        assert_bitwise(got[:, ~m], a[:, ~m], f"case {seed} interior")


def test_gpu_boundary_plan_tiled_level(cx, dev):
    """A level tiled by FABs, conditions drawn at random (some directions
    periodic): one plan launch equals the oracle on every FAB, twice in a
    row (sources are never written, so a second execution changes nothing)."""
    import carpetx_b200 as cb
    from carpetx_b200.workloads import boundary_spec, tiled_level_fabs
    for seed in range(6):
        rng = np.random.default_rng(300 + seed)
        it = tuple(int(v) for v in rng.integers(0, 2, 3))
        ncomp = int(rng.integers(1, 17))
        per = (seed == 3, False, seed == 5)
        spec = boundary_spec(rng, ncomp, it, (24, 16, 20), nghost=3, periodic=per)
        fabs = tiled_level_fabs((24, 16, 20), (8, 8, 4), it, 3)
        host = [fab_data(10 * seed + i, ncomp, lo, hi) for i, (lo, hi) in enumerate(fabs)]
        dev_t = [_dev(a, dev) for a in host]
        plan = cb.BoundaryPlan(spec, [(t, lo, hi) for t, (lo, hi) in zip(dev_t, fabs)])
        plan.execute()
        plan.execute()
        npts = 0
        for t, a, (lo, hi) in zip(dev_t, host, fabs):
            cx.boundary(spec, a, lo, hi)
            assert_bitwise(t.cpu().numpy(), a, f"level {seed}")
            npts += int(outside_mask(spec, lo, hi).sum())
        st = plan.stats()
        # the plan sets at most the points outside the interior (fewer where
        # a face has no condition)
        assert st["points"] <= npts
        plan.close()


def test_gpu_boundary_plan_bench_level(cx, dev):
    """The benchmark's level at full size (256^3 cells in 512 FABs of 32^3,
    3 ghosts, 16 components, every kind of condition): bit-exact on every
    FAB that touches the boundary; interior FABs are skipped and unchanged."""
    import torch
    import carpetx_b200 as cb
    from carpetx_b200.workloads import BC_LEVEL_FACES, boundary_spec, tiled_level_fabs
    rng = np.random.default_rng(7)
    spec = boundary_spec(rng, 16, (1, 1, 1), (256,) * 3, nghost=3, faces=BC_LEVEL_FACES)
    fabs = tiled_level_fabs((256,) * 3, (32,) * 3, (1, 1, 1), 3)
    slab = torch.empty((len(fabs), 16, 38, 38, 38), dtype=torch.float64, device=dev)
    g = torch.Generator(device=dev)
    g.manual_seed(11)
    slab.uniform_(-1, 1, generator=g)
    before = slab.clone()
    plan = cb.BoundaryPlan(spec, [(slab[i], lo, hi) for i, (lo, hi) in enumerate(fabs)])
    plan.execute()
    torch.cuda.synchronize()
    st = plan.stats()
    touched = npts = 0
    for i, (lo, hi) in enumerate(fabs):
        a = before[i].cpu().numpy()
        m = outside_mask(spec, lo, hi)
        if not m.any():
            assert torch.equal(slab[i], before[i])
            continue
        cx.boundary(spec, a, lo, hi)
        assert_bitwise(slab[i].cpu().numpy(), a, f"FAB {i}")
        touched += 1
        npts += int(m.sum())
    assert touched == 512 - 6 ** 3
    # every FAB's points outside the domain (neighbouring FABs' ghosts overlap
    # along the domain's edges, so this exceeds the shell 262^3 - 256^3)
    assert st["points"] == npts


def test_gpu_boundary_rejects(dev):
    import torch
    import carpetx_b200 as cb
    from carpetx_b200.workloads import boundary_spec
    lo, hi = (-2, -2, -2), (7, 7, 7)
    t = torch.zeros((1, 10, 10, 10), dtype=torch.float64, device=dev)
    faces = [[(0, 1), (0, 0), (0, 0)], [(0, 0)] * 3]  # symmetry_boundary alone
    spec = boundary_spec(np.random.default_rng(0), 1, (1, 1, 1), (6, 6, 6), nghost=2, faces=faces)
    with pytest.raises(cb.CxError) as e:
        cb.boundary_box(spec, t, lo, hi)
    assert e.value.status == cb.CX_EINVAL
    with pytest.raises(cb.CxError):
        cb.BoundaryPlan(spec, [(t, lo, hi)])
    faces = [[(3, 0), (0, 0), (0, 0)], [(0, 0)] * 3]
    spec = boundary_spec(np.random.default_rng(0), 1, (1, 1, 1), (1, 6, 6), nghost=2, faces=faces)
    with pytest.raises(cb.CxError):  # a one-cell domain: mirror points leave the interior
        cb.boundary_box(spec, t, lo, hi)
    torch.cuda.synchronize()
    assert not t.any()
