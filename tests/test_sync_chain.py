"""The fine-level ghost sync as one chain (tests/sync_chain.py): on the host
with the oracles, a known answer on linear data; on the GPU with the plans,
bit-identical to the host chain on random data."""
import numpy as np
import pytest

import sync_chain as sc
from helpers import assert_bitwise


def test_sync_chain_oracle_linear(cx):
    """Linear data: every fine ghost point at least two fine cells inside the
    domain holds the linear function's value (from a neighbour or from the
    conservative order-1 prolongation, which reproduces linear cell averages
    exactly; nearer the faces the coarse stencil reads ghosts set by the
    boundary conditions); outside the domain the Dirichlet face holds its
    value."""
    out = sc.oracle_chain(cx, 3, linear=True)
    coarse, fine, _ = sc.level_layout()
    _, fs = sc.specs(3)
    for a, (lo, hi, vlo, vhi) in zip(out, fine):
        z, y, x = np.meshgrid(*[(np.arange(lo[d], hi[d] + 1) + 0.5) * 0.5 for d in (2, 1, 0)],
                              indexing="ij")
        f = 0.125 + 0.25 * x - 0.125 * y + 0.5 * z
        zi, yi, xi = np.meshgrid(*[np.arange(lo[d], hi[d] + 1) for d in (2, 1, 0)], indexing="ij")
        inside = (xi >= 2) & (xi < 30) & (yi >= 2) & (yi < 30) & (zi >= 2) & (zi < 30)
        for c in range(sc.NCOMP):
            assert np.array_equal(a[c][inside], (f + c)[inside])
        # x upper, y lower and z upper are Dirichlet; the fine FABs reach
        # outside the domain only on the lower faces: y lower is Dirichlet
        ylow = (yi < 0) & (xi >= 0) & (xi < 32) & (zi >= 0) & (zi < 32)
        for c in range(sc.NCOMP):
            assert (a[c][ylow] == fs["dirichlet"][c]).all()
        assert not np.isnan(a).any()


def test_sync_chain_layout_patches_disjoint():
    coarse, fine, patches = sc.level_layout()
    for i, (lo, hi, vlo, vhi) in enumerate(fine):
        seen = np.zeros(sc.shape(lo, hi), int)
        for j, (plo, phi) in patches:
            if j != i:
                continue
            sl = tuple(slice(plo[d] - lo[d], phi[d] - lo[d] + 1) for d in (2, 1, 0))
            seen[sl] += 1
        assert seen.max() == 1


@pytest.mark.gpu
def test_gpu_sync_chain_matches_oracle(cx, dev):
    want = sc.oracle_chain(cx, 11)
    got = sc.gpu_chain(cx, 11, dev)
    for i, (g, w) in enumerate(zip(got, want)):
        assert_bitwise(g, w, f"fine FAB {i}")


@pytest.mark.gpu
def test_gpu_sync_chain_graph_replay(cx, dev):
    """The six plan executions of a sync captured into one CUDA graph and
    replayed twice give the host chain's result bit for bit."""
    want = sc.oracle_chain(cx, 12)
    got = sc.gpu_chain(cx, 12, dev, graph=True)
    for i, (g, w) in enumerate(zip(got, want)):
        assert_bitwise(g, w, f"fine FAB {i}")
