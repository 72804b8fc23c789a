"""Coarse-patch gather of a distributed level transfer: the piece list, and
the exchange itself run as two gloo ranks on the CPU, checked point by point
against the coarse level's values."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

import carpetx_b200 as cb
from carpetx_b200.distribute import box_cost, knapsack
from carpetx_b200.fillpatch import CoarsePatchExchange, intersect, patch_pieces


def coarse_level():
    """A 32 x 24 x 16 coarse domain cut into 8 x 8 x 8 boxes, with ranks."""
    boxes = [((i, j, k), (i + 7, j + 7, k + 7)) for k in (0, 8) for j in (0, 8, 16)
             for i in (0, 8, 16, 24)]
    return boxes


def fine_patches(seed, op_spec=("interpolate", 3, 0), n=10):
    """Coarse patches (CoarseBox of the fine regions) of random fine boxes of
    the refined domain, some reaching past the coarse domain."""
    rng = np.random.default_rng(seed)
    op = cb.Op(*op_spec)
    out = []
    for _ in range(n):
        flo = tuple(int(v) for v in rng.integers(-4, [60, 44, 28]))
        fhi = tuple(flo[d] + int(rng.integers(4, 24)) for d in range(3))
        out.append(op.coarse_box(flo, fhi))
    return out


def value(c, i, j, k):
    return float(i + 100 * j + 10000 * k + 1e6 * c)


def box_values(box, ncomp):
    lo, hi = box
    k, j, i = np.meshgrid(*[np.arange(lo[d], hi[d] + 1) for d in (2, 1, 0)], indexing="ij")
    return np.stack([i + 100 * j + 10000 * k + 1e6 * c for c in range(ncomp)]).astype(np.float64)


def test_intersect():
    assert intersect(((0, 0, 0), (3, 3, 3)), ((2, 1, 3), (9, 9, 9))) == ((2, 1, 3), (3, 3, 3))
    assert intersect(((0, 0, 0), (3, 3, 3)), ((4, 0, 0), (5, 5, 5))) is None


def test_pieces_tile_each_patch():
    coarse = coarse_level()
    patches = fine_patches(1)
    pieces = patch_pieces(coarse, [0] * len(coarse), patches, [0] * len(patches))
    domain = ((0, 0, 0), (31, 23, 15))
    for pi, pb in enumerate(patches):
        cover = np.zeros(tuple(pb[1][d] - pb[0][d] + 1 for d in (2, 1, 0)), int)
        for _, _, _, q, piece in pieces:
            if q != pi:
                continue
            cover[piece[0][2] - pb[0][2]:piece[1][2] - pb[0][2] + 1,
                  piece[0][1] - pb[0][1]:piece[1][1] - pb[0][1] + 1,
                  piece[0][0] - pb[0][0]:piece[1][0] - pb[0][0] + 1] += 1
        inside = intersect(pb, domain)
        want = np.zeros_like(cover)
        if inside:
            want[inside[0][2] - pb[0][2]:inside[1][2] - pb[0][2] + 1,
                 inside[0][1] - pb[0][1]:inside[1][1] - pb[0][1] + 1,
                 inside[0][0] - pb[0][0]:inside[1][0] - pb[0][0] + 1] = 1
        assert np.array_equal(cover, want), "pieces must tile the patch inside the domain once"
    # the same sorted list for any rank
    assert pieces == sorted(pieces, key=lambda t: t[:4])


def test_single_rank_exchange_copies_locally():
    coarse = coarse_level()
    patches = fine_patches(2)
    ex = CoarsePatchExchange(coarse, [0] * len(coarse), patches, [0] * len(patches), 0)
    cdata = {i: torch.from_numpy(box_values(b, 2)) for i, b in enumerate(coarse)}
    pdata = {i: torch.full((2,) + tuple(b[1][d] - b[0][d] + 1 for d in (2, 1, 0)), float("nan"),
                           dtype=torch.float64) for i, b in enumerate(patches)}
    ex.run(cdata, pdata)
    check_patches(patches, pdata, 2)
    assert ex.stats()["send"] == 0 and ex.stats()["recv"] == 0


def check_patches(patches, pdata, ncomp):
    domain = ((0, 0, 0), (31, 23, 15))
    for i, b in pdata.items():
        got = b.numpy()
        want = box_values(patches[i], ncomp)
        inside = intersect(patches[i], domain)
        mask = np.zeros(got.shape[1:], bool)
        if inside:
            lo = patches[i][0]
            mask[inside[0][2] - lo[2]:inside[1][2] - lo[2] + 1,
                 inside[0][1] - lo[1]:inside[1][1] - lo[1] + 1,
                 inside[0][0] - lo[0]:inside[1][0] - lo[0] + 1] = True
        assert np.array_equal(got[:, mask], want[:, mask]), f"patch {i}"
        assert np.all(np.isnan(got[:, ~mask])), f"patch {i}: uncovered points were written"


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        coarse = coarse_level()
        patches = fine_patches(3, n=14)
        # the coarse level and the fine level are distributed independently
        cown = knapsack([box_cost(b[0], b[1], 1) for b in coarse], world)
        cown = [(r + 1) % world for r in cown]  # a different mapping from the fine one
        pown = knapsack([box_cost(b[0], b[1], 1) for b in patches], world)
        ex = CoarsePatchExchange(coarse, cown, patches, pown, rank)
        st = ex.stats()
        assert st["send"] > 0 and st["recv"] > 0, "the test must exercise the exchange"
        ncomp = 3
        cdata = {i: torch.from_numpy(box_values(b, ncomp)) for i, b in enumerate(coarse)
                 if cown[i] == rank}
        pdata = {i: torch.full((ncomp,) + tuple(b[1][d] - b[0][d] + 1 for d in (2, 1, 0)),
                               float("nan"), dtype=torch.float64)
                 for i, b in enumerate(patches) if pown[i] == rank}
        ex.run(cdata, pdata)
        check_patches(patches, pdata, ncomp)
        # a second exchange on the same plan (the per-step sync repeats it)
        for t in cdata.values():
            t.mul_(2.0)
        ex.run(cdata, pdata)
        for i, t in pdata.items():
            assert np.allclose(np.nan_to_num(t.numpy()), 2 * np.nan_to_num(
                box_values(patches[i], ncomp) * ~np.isnan(t.numpy())))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_two_gloo_ranks_gather_coarse_patches(world):
    mp.start_processes(_rank_main, args=(world, _free_port()), nprocs=world, join=True,
                       start_method="spawn")


@pytest.mark.gpu
def test_gpu_exchange_local_copy_plan_matches_tensor_copies(dev):
    """One rank owning everything: the local pieces go through one copy-plan
    launch on CUDA tensors and through one tensor copy each on CPU tensors;
    vertex-centred coarse boxes overlap on shared faces with different
    values there, so the order in which sources win is exercised too."""
    rng = np.random.default_rng(8)
    coarse = [((i, j, k), (i + 8, j + 8, k + 8)) for k in (0, 8) for j in (0, 8, 16)
              for i in (0, 8, 16, 24)]  # shared faces
    patches = fine_patches(3, ("interpolate", 3, 0), n=12)
    ex = CoarsePatchExchange(coarse, [0] * len(coarse), patches, [0] * len(patches), 0)
    shape = lambda b: tuple(b[1][d] - b[0][d] + 1 for d in (2, 1, 0))  # noqa: E731
    cdat = {ci: rng.uniform(-1, 1, (2,) + shape(b)) for ci, b in enumerate(coarse)}
    host_c = {ci: torch.from_numpy(a) for ci, a in cdat.items()}
    host_p = {pi: torch.full((2,) + shape(b), np.nan, dtype=torch.float64)
              for pi, b in enumerate(patches)}
    dev_c = {ci: t.to(dev) for ci, t in host_c.items()}
    dev_p = {pi: t.to(dev) for pi, t in host_p.items()}
    ex.run(host_c, host_p)
    ex.run(dev_c, dev_p)
    assert ex._plan is not None
    for pi in host_p:
        a, b = host_p[pi].numpy(), dev_p[pi].cpu().numpy()
        assert np.array_equal(a.view(np.uint64), b.view(np.uint64)), f"patch {pi}"
