"""The package's sync chain (carpetx_b200.sync.SyncChain), with and without
the prolongation writing the fine patches into the fine FABs directly (no
patch buffers, no scatter), on the layout of tests/sync_chain.py: both are
bit-identical to the host chain of the oracles, also from one CUDA graph."""
import pytest
import torch

import carpetx_b200 as cb
import sync_chain as sc
from helpers import assert_bitwise

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("fused", [False, True])
def test_gpu_package_sync_chain_matches_oracle(cx, dev, fused):
    from carpetx_b200.sync import SyncChain
    want = sc.oracle_chain(cx, 13)
    coarse, fine, patches = sc.level_layout()
    cs, fs = sc.specs(13)
    ca, fa = sc.initial_data(13, coarse, fine)
    gc = [(torch.from_numpy(a).to(dev),) + tuple(b) for a, b in zip(ca, coarse)]
    gf = [(torch.from_numpy(a).to(dev),) + tuple(b) for a, b in zip(fa, fine)]
    chain = SyncChain(cb.Op(*sc.OP), sc.NCOMP, gc, gf, sc.NG, cs, fs, fused=fused)
    assert [name for name, _ in chain.steps] == (
        ["fill_boundary", "gather", "coarse_bc", "prolong", "fine_bc"] if fused else
        ["fill_boundary", "gather", "coarse_bc", "prolong", "scatter", "fine_bc"])
    assert len(chain.patches) == len(patches)
    chain.execute()
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        chain.execute()
    g.replay()
    torch.cuda.synchronize()
    del g
    for i, (f, w) in enumerate(zip(gf, want)):
        assert_bitwise(f[0].cpu().numpy(), w, f"fine FAB {i} (fused={fused})")
    chain.close()


@pytest.mark.parametrize("op,wide", [(sc.OP, False), (("hermite", 3, 7), False), (sc.OP, True)])
def test_gpu_package_sync_chain_direct_matches_oracle(cx, dev, op, wide):
    """direct=True: the fine patches whose coarse box lies in one coarse FAB
    read that FAB (its ghosts synced first, as the level loop has them),
    patches spanning coarse FABs are cut where every piece then fits, the
    rest are gathered; bit-identical to the host chain of the oracles, which
    gathers every patch from the coarse valid boxes.  Cases: every patch
    direct and whole; hermite o3, whose reach outside the domain exceeds the
    coarse ghosts, with both kinds; one wide fine FAB, whose patches are
    cut."""
    from carpetx_b200.sync import SyncChain
    want = sc.oracle_chain(cx, 13, op=op, wide=wide)
    coarse, fine, patches = sc.level_layout(wide)
    cs, fs = sc.specs(13)
    ca, fa = sc.initial_data(13, coarse, fine)
    gc = [(torch.from_numpy(a).to(dev),) + tuple(b) for a, b in zip(ca, coarse)]
    gf = [(torch.from_numpy(a).to(dev),) + tuple(b) for a, b in zip(fa, fine)]
    # the coarse level's own sync: its halo exchange, then its boundary conditions
    cfill = cb.CopyPlan.fill_boundary(gc, sc.NCOMP, sc.NG)
    cbc = cb.BoundaryPlan(cs, [g[:3] for g in gc])
    cfill.execute()
    cbc.execute()
    chain = SyncChain(cb.Op(*op), sc.NCOMP, gc, gf, sc.NG, cs, fs, direct=True)
    ndirect = sum(s is not None for s in chain.src)
    assert 0 < ndirect <= len(chain.patches)
    assert (len(chain.patches) > len(patches)) == wide  # cut pieces
    assert (ndirect < len(chain.patches)) == (op != sc.OP)  # gathered patches
    names = [name for name, _ in chain.steps]
    assert names[0] == "fill_boundary" and names[-2:] == ["prolong", "fine_bc"]
    assert ("gather" in names) == (ndirect < len(chain.patches))
    chain.execute()
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        chain.execute()
    g.replay()
    torch.cuda.synchronize()
    del g
    for i, (f, w) in enumerate(zip(gf, want)):
        assert_bitwise(f[0].cpu().numpy(), w, f"fine FAB {i} (direct, {op}, wide={wide})")
    chain.close()
    cfill.close()
    cbc.close()
