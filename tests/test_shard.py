"""Sharding a batch over ranks: the partition (CPU) and the collectives the
multi-GPU benchmark uses, run as two `gloo` ranks on CPU."""
import os
import socket

import pytest

import shard


def test_lpt_partition_is_disjoint_complete_and_balanced():
    import workloads as W
    entries = W.batch_entries(4096, 8, 18, seed=0)
    costs = [W.est_interactions(k, d) for k, d, _ in entries]
    for world in (1, 2, 4, 8):
        parts = shard.lpt_partition(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(entries)))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(costs)  # the LPT bound
        assert parts == shard.lpt_partition(costs, world)  # deterministic


def test_lpt_partition_edge_cases():
    assert shard.lpt_partition([], 3) == [[], [], []]
    assert shard.lpt_partition([5.0], 2) == [[0], []]
    with pytest.raises(ValueError):
        shard.lpt_partition([1.0], 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    import workloads as W
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        entries = W.batch_entries(256, 4, 12, seed=0)
        mine = shard.rank_share(entries, lambda e: W.est_interactions(e[0], e[1]), rank, world)
        # stand-in for this rank's reduction: predicted interactions per net
        results = [(j, W.est_interactions(k, d)) for k, d, j in mine]
        work = sum(r for _, r in results)
        slowest = shard.max_over_ranks(work, dist, "cpu")
        total = shard.sum_over_ranks(work, dist, "cpu")
        got = shard.gather_to_root(results, dist, rank, world)
        if rank == 0:
            flat = sorted(j for part in got for j, _ in part)
            q.put(("ok", flat == sorted(j for _, _, j in entries), slowest, total,
                   sum(W.est_interactions(k, d) for k, d, _ in entries)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_share_and_gather():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs)
    tag, complete, slowest, total, want = q.get(timeout=10)
    assert complete
    assert abs(total - want) < 1e-6 * want
    assert want / 2 <= slowest <= want / 2 + max(1.0, want * 0.05)
