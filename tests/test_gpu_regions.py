"""GPU tests of the copy plans (cx_copy_plan_fill_boundary,
cx_copy_plan_parallel_copy) against the numpy restatement of AMReX's
FillBoundary and ParallelCopy (oracle/regions.py): bit-exact on every point,
with random data (where valid boxes share vertex faces the values differ, so
the first-source rule is exercised) and with known values on the benchmark's
level."""
import numpy as np
import pytest

from region_cases import in_domain, known_value, random_patches, tiled, valid_mask
from oracle import regions

pytestmark = pytest.mark.gpu


def _to_dev(fabs, dev):
    import torch
    return [(torch.from_numpy(f[0]).to(dev), f[1], f[2], f[3], f[4]) for f in fabs]


def _random_level(rng, domain_n, box_n, it, ng, ncomp):
    out = []
    for lo, hi, vlo, vhi in tiled(domain_n, box_n, it, ng):
        shape = tuple(hi[d] - lo[d] + 1 for d in (2, 1, 0))
        out.append([rng.uniform(-1, 1, (ncomp,) + shape), lo, hi, vlo, vhi])
    return out


@pytest.mark.parametrize("it", [(1, 1, 1), (0, 0, 0), (1, 0, 1)])
@pytest.mark.parametrize("periodic", [(0, 0, 0), (1, 1, 1), (1, 0, 0)])
def test_gpu_fill_boundary_matches_oracle(dev, it, periodic):
    import carpetx_b200 as cb
    dn, bn, ng = (12, 8, 8), (4, 4, 8), (2, 3, 1)
    period = tuple(dn[d] if periodic[d] else 0 for d in range(3))
    host = _random_level(np.random.default_rng(sum(it) + 3 * sum(periodic)), dn, bn, it, ng, 2)
    gpu = _to_dev(host, dev)
    plan = cb.CopyPlan.fill_boundary(gpu, 2, ng, period)
    plan.execute()
    plan.execute()  # sources are valid points, never written: a no-op
    regions.fill_boundary(host, ng, period)
    for g, h in zip(gpu, host):
        assert np.array_equal(g[0].cpu().numpy().view(np.uint64), h[0].view(np.uint64))
    plan.close()


@pytest.mark.parametrize("src_ng,dst_ng,period", [((0, 0, 0), (1, 1, 1), (16, 0, 0)),
                                                  ((1, 1, 1), (2, 2, 2), (16, 16, 8)),
                                                  ((0, 0, 0), (0, 0, 0), (0, 0, 0))])
def test_gpu_parallel_copy_matches_oracle(dev, src_ng, dst_ng, period):
    import carpetx_b200 as cb
    rng = np.random.default_rng(9)
    src = _random_level(rng, (16, 16, 8), (8, 4, 8), (1, 1, 1), (1, 1, 1), 3)
    dst = random_patches(np.random.default_rng(4), 6, (16, 16, 8), 3)
    g_src, g_dst = _to_dev(src, dev), _to_dev(dst, dev)
    plan = cb.CopyPlan.parallel_copy(g_dst, g_src, 3, src_ng, dst_ng, period)
    plan.execute()
    regions.parallel_copy(dst, src, src_ng, dst_ng, period)
    for g, h in zip(g_dst, dst):
        assert np.array_equal(g[0].cpu().numpy().view(np.uint64), h[0].view(np.uint64))
    plan.close()


def test_gpu_fill_boundary_bench_level(dev):
    """The benchmark's level (512 FABs of 32^3 cells + 3 ghosts, 16
    components, not periodic): after one launch every ghost point inside the
    domain holds its index's value and every point outside it is untouched."""
    import torch
    import carpetx_b200 as cb
    ng, n = (3, 3, 3), 256
    fabs = tiled((n,) * 3, (32,) * 3, (1, 1, 1), ng)
    slab = torch.empty((len(fabs), 16, 38, 38, 38), dtype=torch.float64, device=dev)
    m_valid = torch.from_numpy(valid_mask(fabs[0][0], fabs[0][1], fabs[0][2], fabs[0][3])).to(dev)
    for i, (lo, hi, vlo, vhi) in enumerate(fabs):
        slab[i] = torch.from_numpy(known_value(16, lo, hi, (0, 0, 0))).to(dev)
        slab[i][:, ~m_valid] = float("nan")
    plan = cb.CopyPlan.fill_boundary([(slab[i],) + f for i, f in enumerate(fabs)], 16, ng)
    st = plan.stats()
    plan.execute()
    torch.cuda.synchronize()
    filled = 0
    for i, (lo, hi, vlo, vhi) in enumerate(fabs):
        want = torch.from_numpy(known_value(16, lo, hi, (0, 0, 0))).to(dev)
        m = torch.from_numpy(in_domain(lo, hi, (0, 0, 0), (n - 1,) * 3, (0, 0, 0))).to(dev)
        assert torch.equal(slab[i][:, m], want[:, m]), f"FAB {i}"
        assert torch.isnan(slab[i][:, ~m]).all(), f"FAB {i}"
        filled += int((m & ~m_valid).sum())
    assert st["points"] == filled
    plan.close()


def test_gpu_copy_plan_rejects(dev):
    import torch
    import carpetx_b200 as cb
    t = torch.zeros((1, 5, 5, 5), dtype=torch.float64, device=dev)
    with pytest.raises(cb.CxError) as e:
        cb.CopyPlan.fill_boundary([(t, (0, 0, 0), (4, 4, 4), (1, 1, 1), (5, 3, 3))], 1,
                                  (1, 1, 1))
    assert e.value.status == cb.CX_EINVAL
    assert not t.any()
