"""Host logic of the multi-GPU path (one process per GPU): the knapsack
distribution of a level's boxes over ranks, and the max / sum reductions the
benchmark times with, run as two gloo ranks on the CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from carpetx_b200.distribute import (box_cost, knapsack, max_over_ranks, my_boxes, rank_loads,
                                     sum_over_ranks)
from carpetx_b200.workloads import mixed_level_boxes


def level(nboxes, seed=2026, ncomp=24):
    boxes = [(it, clo, chi, flo, fhi, ncomp) for it, clo, chi, flo, fhi in
             mixed_level_boxes(seed, nboxes=nboxes)]
    return boxes, [box_cost(b[3], b[4], b[5]) for b in boxes]


def test_box_cost():
    assert box_cost((0, 0, 0), (7, 3, 1), 5) == 8 * 4 * 2 * 5
    assert box_cost((0, 0, 0), (-1, 3, 1), 5) == 0


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_knapsack_covers_and_balances(world):
    boxes, costs = level(512 * world)
    owner = knapsack(costs, world)
    assert len(owner) == len(boxes) and set(owner) <= set(range(world))
    loads = rank_loads(costs, owner, world)
    assert sum(loads) == sum(costs)
    # longest-processing-time: every rank within the largest box of the mean
    mean = sum(costs) / world
    assert max(loads) <= mean + max(costs)
    assert max(loads) / mean < 1.001
    # a pure function of the box list
    assert knapsack(costs, world) == owner


def test_knapsack_edge_cases():
    assert knapsack([], 3) == []
    assert knapsack([5], 4) == [0]
    assert knapsack([1, 1, 1, 1], 2) == [0, 1, 0, 1]
    assert rank_loads([3, 2, 2], knapsack([3, 2, 2], 2), 2) == [3, 4]
    with pytest.raises(ValueError):
        knapsack([1], 0)


def test_reductions_without_process_group():
    assert max_over_ranks(2.5) == 2.5
    assert sum_over_ranks(2.5) == 2.5


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, nboxes):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        boxes, costs = level(nboxes)
        mine = my_boxes(boxes, costs, rank, world)
        # every rank computed the same mapping: the parts are disjoint and
        # cover the level
        parts = [None] * world
        dist.all_gather_object(parts, mine)
        seen = [b for p in parts for b in p]
        assert sorted(seen) == sorted(boxes)
        assert parts[rank] == mine
        owner = knapsack(costs, world)
        for r in range(world):
            assert parts[r] == [b for b, o in zip(boxes, owner) if o == r]
        # the benchmark's timing reductions
        assert max_over_ranks(float(rank + 1)) == float(world)
        assert sum_over_ranks(float(rank + 1)) == world * (world + 1) / 2
        work = sum(box_cost(b[3], b[4], b[5]) for b in mine)
        assert sum_over_ranks(work) == sum(costs)
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_two_gloo_ranks_share_a_level(world):
    port = _free_port()
    mp.start_processes(_rank_main, args=(world, port, 1024), nprocs=world, join=True,
                       start_method="spawn")
