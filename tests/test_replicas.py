"""Replica parallelism (one process per GPU, independent materials): the cost-model partition
and the host-side exchange, run as two gloo ranks on the CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from openntc_b200.replicas import MaterialSpec, ReplicaGroup, partition, run_share


def batch_of_16():
    """A mixed batch like the 16-material configuration: 256^2..4096^2, C in {4, 6, 9, 12}, all profiles."""
    dims = [256, 512, 1024, 2048, 4096]
    chans = [4, 6, 9, 12]
    return [MaterialSpec(f"m{i}", dims[i % 5], chans[i % 4], i % 4, 2000 + 250 * (i % 3), 1 + i % 2) for i in range(16)]


def test_partition_covers_every_item_once_and_balances():
    specs = batch_of_16()
    costs = [s.cost() for s in specs]
    for world in (1, 2, 3, 4, 8, 16, 20):
        parts = partition(costs, world)
        assert len(parts) == world
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(specs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        # longest-processing-time bound: no rank exceeds the lightest by more than the largest item
        assert max(loads) - min(loads) <= max(costs) + 1e-6
    assert partition(costs, 4) == partition(costs, 4)  # deterministic


def test_partition_edge_cases():
    assert partition([], 3) == [[], [], []]
    assert partition([5.0], 2) == [[0], []]
    with pytest.raises(ValueError):
        partition([1.0], 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank))
    g = ReplicaGroup(world, rank, backend="gloo", timeout_s=60)
    try:
        specs = batch_of_16()
        done = []

        def work(spec):
            done.append(spec.name)
            return {"rank": rank, "cost": spec.cost()}

        results = run_share(specs, g, work)
        slowest = g.max(float(10 + rank))
        g.barrier()
        q.put((rank, sorted(done), results, slowest))
    finally:
        g.close()


def test_two_gloo_ranks_train_disjoint_shares_and_exchange_results():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    names = [n for _, done, _, _ in out for n in done]
    assert sorted(names) == sorted(s.name for s in batch_of_16())  # every material once
    assert not set(out[0][1]) & set(out[1][1])
    for rank, done, results, slowest in out:
        assert slowest == 11.0                                      # max over ranks
        assert set(results) == {s.name for s in batch_of_16()}      # every rank sees all results
        assert all(results[n]["rank"] == rank for n in done)
