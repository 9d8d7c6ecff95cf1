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
    return [c["nx"] * c["ny"] * (c["nx"] * c["ny"]) ** 0.4 for c in cases]


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
