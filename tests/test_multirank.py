"""Multi-rank path of bench.py on CPU with gloo (world size 2).

The path shards by independent disorder samples: every rank runs its own
samples (weak scaling) and the only cross-rank operations are a barrier and
the max of the timings.  Checked here: the shards are disjoint and complete,
and the MAX reduction bench.py applies gives the slowest rank's time.
"""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    Ns, seeds = bench.workload(256, rank)
    gathered = [None] * world
    dist.all_gather_object(gathered, (Ns, seeds))
    t = torch.tensor([10.0 + rank])
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.barrier()
    if rank == 0:
        q.put((gathered, float(t.item())))
    dist.destroy_process_group()


def _shard_worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    import cuda_pspin_b200 as ps
    Ns, seeds = bench.workload(256, 0)                  # one fixed set of samples for all ranks
    of = ps.shard_samples(Ns, 96, world)
    mine = [int(k) for k in range(len(Ns)) if of[k] == rank]
    gathered = [None] * world
    dist.all_gather_object(gathered, mine)
    dist.barrier()
    if rank == 0:
        q.put((gathered, Ns))
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_fixed_samples_shard_by_cost(world):
    """A fixed set of samples of uneven N spread over `world` ranks by
    pspin_shard_samples (no communication: every rank computes the same
    assignment): every sample on exactly one rank, and the ranks' N^4 costs
    within the largest single sample's cost of each other."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    gathered, Ns = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    allk = sorted(k for g in gathered for k in g)
    assert allk == list(range(len(Ns)))
    loads = [sum(Ns[k] ** 4 for k in g) for g in gathered]
    assert max(loads) - min(loads) <= max(Ns) ** 4


def test_sample_sharding_and_max_timing():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    gathered, tmax = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (N0, s0), (N1, s1) = gathered
    assert N0 == N1                          # same N mix on every rank
    assert not set(s0) & set(s1)             # disjoint disorder samples
    assert sorted(s0 + s1) == list(range(1000, 1000 + 512))
    assert tmax == 11.0                      # the slowest rank's time
    assert sorted(set(N0)) == [24, 32, 48, 64]
