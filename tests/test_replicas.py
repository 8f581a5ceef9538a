"""Multi-rank host logic on the CPU: partitioning of independent scenarios
over ranks and the timing reductions, with world-size-2 gloo process groups
(127.0.0.1 rendezvous).  No GPU."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from loquat_b200 import replicas


def test_partition_covers_every_unit_once_and_balances():
    rng = np.random.default_rng(0)
    counts = np.exp(rng.uniform(np.log(5e3), np.log(2e5), 256))
    for world in (1, 2, 3, 4, 8):
        shares = replicas.partition(counts, world)
        flat = sorted(k for s in shares for k in s)
        assert flat == list(range(256))
        assert len(shares) == world
        assert replicas.imbalance(counts, shares) < 1.02
    assert replicas.partition([], 2) == [[], []]
    with pytest.raises(ValueError):
        replicas.partition([1.0], 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, counts, out):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        shares = replicas.partition(counts, world)
        mine = shares[rank]
        # each rank "times" its share as its particle count; the job time is the max
        t = float(sum(counts[k] for k in mine))
        out[rank] = (replicas.max_over_ranks(t), replicas.sum_over_ranks(len(mine)), mine)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_split_an_ensemble_and_reduce_times():
    world = 2
    counts = [5e3, 2e5, 7e4, 1.2e4, 9e4, 3e4, 1.5e5, 6e3]
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_worker, args=(r, world, port, counts, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    shares = replicas.partition(counts, world)
    loads = [sum(counts[k] for k in s) for s in shares]
    for r in range(world):
        tmax, nsum, mine = out[r]
        assert tmax == max(loads)
        assert nsum == len(counts)
        assert mine == shares[r]
    assert sorted(out[0][2] + out[1][2]) == list(range(len(counts)))


def test_reductions_without_a_process_group_are_identity():
    assert replicas.max_over_ranks(3.5) == 3.5
    assert replicas.sum_over_ranks(2.0) == 2.0
