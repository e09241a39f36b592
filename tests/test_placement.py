"""Placement of independent grids across ranks, and the host reductions of the N > 1 path,
run as world-size-2 gloo process groups on the CPU."""
import os
import socket

import numpy as np
import pytest


def test_place_is_balanced_and_within_budget():
    from fluidsim_b200.placement import mine, place

    rng = np.random.default_rng(0)
    cells = [int(rng.integers(64, 1024)) ** 2 for _ in range(256)]
    sizes = [160 * c for c in cells]
    world = 8
    budget = sum(sizes)  # generous: balance decides
    a = place(cells, sizes, world, budget)
    assert sorted(i for r in range(world) for i in mine(a, r)) == list(range(256))
    load = [sum(cells[i] for i in mine(a, r)) for r in range(world)]
    assert max(load) - min(load) <= max(cells)
    assert a == place(cells, sizes, world, budget)  # deterministic


def test_place_respects_budget_and_rejects_misfits():
    from fluidsim_b200.placement import place

    a = place([10, 9, 8, 1], [10, 9, 8, 1], 2, 19)
    used = [sum(s for s, r in zip([10, 9, 8, 1], a) if r == k) for k in range(2)]
    assert max(used) <= 19 and a == [0, 1, 1, 0]
    # The least-loaded rank is full: the grid goes to the one with room.
    assert place([10, 1, 9], [10, 10, 1], 2, 11) == [0, 1, 1]
    with pytest.raises(ValueError):
        place([5, 5], [20, 1], 2, 10)
    with pytest.raises(ValueError):
        place([1], [1], 0, 10)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist

    from fluidsim_b200.placement import max_over_ranks, mine, place, sum_over_ranks

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        cells = [(64 + 37 * k) ** 2 for k in range(23)]
        a = place(cells, [8 * c for c in cells], world, 10**12)
        local = mine(a, rank)
        # Every rank's share, its slowest "time" and the total work, agreed over the group.
        slowest = max_over_ranks(1.0 + rank)
        total = sum_over_ranks(sum(cells[i] for i in local))
        out.put((rank, local, slowest, total, sum(cells)))
    finally:
        dist.destroy_process_group()


def test_two_ranks_share_the_grids_without_overlap():
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    results.sort()
    shares = [set(r[1]) for r in results]
    assert not (shares[0] & shares[1]) and shares[0] | shares[1] == set(range(23))
    for _, _, slowest, total, expect in results:
        assert slowest == 2.0 and total == expect
