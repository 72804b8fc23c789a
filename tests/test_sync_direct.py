"""Host logic of the sync chain's direct mode (carpetx_b200.sync):
split_at cuts a box into a partition, and direct_sources picks, per piece of
the fine patches, a coarse FAB whose box holds the piece's coarse box (or
none: gathered), cutting a patch only where every piece then fits."""
import itertools

import numpy as np
import pytest

import carpetx_b200 as cb
import sync_chain as sc
from carpetx_b200.sync import direct_sources, fine_patches, split_at


def _cells(box):
    lo, hi = box
    return {c for c in itertools.product(*[range(lo[d], hi[d] + 1) for d in range(3)])}


def test_split_at_partitions():
    rng = np.random.default_rng(3)
    for _ in range(50):
        lo = tuple(int(v) for v in rng.integers(-5, 5, 3))
        hi = tuple(lo[d] + int(rng.integers(0, 7)) for d in range(3))
        cuts = [sorted(set(int(v) for v in rng.integers(-6, 13, int(rng.integers(0, 4)))))
                for _ in range(3)]
        pieces = split_at((lo, hi), cuts)
        seen = set()
        for p in pieces:
            c = _cells(p)
            assert not (c & seen)
            seen |= c
            for d in range(3):  # no cut strictly inside a piece
                assert not any(p[0][d] < x <= p[1][d] for x in cuts[d])
        assert seen == _cells((lo, hi))


@pytest.mark.parametrize("op,wide,want", [
    (sc.OP, False, (18, 18, 0)),               # every patch whole from one FAB
    (("hermite", 3, 7), False, (18, 4, 0)),    # reach outside the domain: 14 gathered
    (sc.OP, True, (18, 18, 4)),                # a wide fine FAB: 4 patches cut
])
def test_direct_sources(op, wide, want):
    coarse, fine, _ = sc.level_layout(wide)
    o = cb.Op(*op)
    patches = fine_patches(fine)
    pieces, src = direct_sources(o, coarse, patches)
    ncut = len([1 for i, p in patches if (i, p) not in pieces])
    assert (len(pieces), sum(s is not None for s in src), ncut) == want
    # the pieces of each FAB partition its patches
    for f in range(len(fine)):
        a = set().union(*[_cells(p) for i, p in patches if i == f])
        b = [_cells(p) for i, p in pieces if i == f]
        assert sum(len(x) for x in b) == len(a) and set().union(*b) == a
    # a chosen FAB holds the piece's coarse box
    for (i, p), s in zip(pieces, src):
        if s is not None:
            lo, hi = o.coarse_box(p[0], p[1])
            assert all(coarse[s][0][d] <= lo[d] and hi[d] <= coarse[s][1][d] for d in range(3))
