"""Multi-GPU sharding of the batched form, on CPU: every rank computes its own
share with ifc.shard_cases (no data-path collective); two gloo ranks check
that the shares are disjoint, cover every case and are balanced, the only
exchange being a gather of the per-rank case lists for the check."""
import os

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import ifc


def weights(cases):
    return [ifc.case_weight(c) for c in cases]


def test_shard_partition_single_process():
    cases = ifc.batch_cases(256, seed=0)
    w = weights(cases)
    for world in (1, 2, 4, 8):
        parts = [ifc.shard_cases(w, r, world) for r in range(world)]
        allidx = sorted(i for p in parts for i in p)
        assert allidx == list(range(256))
        loads = [sum(w[i] for i in p) for p in parts]
        assert max(loads) <= 1.05 * (sum(w) / world) + max(w)


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    cases = ifc.batch_cases(64, seed=1)
    mine = ifc.shard_cases(weights(cases), rank, world)
    gathered = [None] * world
    dist.all_gather_object(gathered, mine)
    if rank == 0:
        q.put(gathered)
    dist.destroy_process_group()


def test_shard_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    gathered = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    a, b = gathered
    assert not set(a) & set(b)
    assert sorted(a + b) == list(range(64))


def _totals_worker(rank, world, port, q):
    """Each rank solves (here: pretends to solve) its share of the batch and
    the bench's cross-rank reduction forms the whole-job line."""
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import torch

    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    cases = ifc.batch_cases(64, seed=1)
    mine = ifc.shard_cases(weights(cases), rank, world)
    local = {"solves": len(mine), "updates": 1000.0 * (rank + 1), "case_its": 10 * len(mine),
             "conv_batch": len(mine), "conv_plain": len(mine) - rank, "batch_ms": 5.0 + rank,
             "plain_ms": 40.0 - rank, "worst": 1e-7 * (rank + 1)}
    tot = bench.batch_totals(local, world, torch.device("cpu"))
    if rank == 0:
        q.put(tot)
    dist.destroy_process_group()


def test_batch_totals_two_gloo_ranks():
    """The batch bench's per-rank results gathered end to end on two gloo
    ranks: counts are summed over the ranks, times take the slowest rank."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 30500 + os.getpid() % 1000
    procs = [ctx.Process(target=_totals_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    tot = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert tot["solves"] == 64 and tot["case_its"] == 640
    assert tot["updates"] == 3000.0 and tot["conv_batch"] == 64 and tot["conv_plain"] == 63
    assert tot["batch_ms"] == 6.0 and tot["plain_ms"] == 40.0 and abs(tot["worst"] - 2e-7) < 1e-20
