"""bench.py's multi-rank harness with two gloo ranks on the CPU: the job time is
the slowest rank's, the replica throughput counts every replica's bodies, and the
ensemble's instances are split across the ranks with every instance run exactly
once and the job's body count equal to the whole ensemble's."""
import os
import socket

import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    t = bench.max_over_ranks(1.0 + rank, device="cpu")
    q.put((rank, t, bench.replica_throughput(100, 10, world, t)))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_and_throughput():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [2.0, 2.0]
    assert all(abs(o[2] - 2 * 100 * 10 / 2.0) < 1e-12 for o in out)


def test_single_process_is_identity():
    import bench
    assert bench.max_over_ranks(3.5, device="cpu") == 3.5
    assert bench.replica_throughput(2048, 20, 1, 2.0) == 2048 * 20 / 2.0


def _ensemble_rank(rank, world, port, q):
    import datetime

    import torch
    import torch.distributed as dist

    import bench
    from timstochrigidbodiessim_b200 import configs
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    mine = bench.ensemble_shard(64, rank, world)
    shards = [None] * world
    dist.all_gather_object(shards, mine)
    counts = configs.ensemble_body_counts(64)
    bodies = torch.tensor([float(sum(counts[i] for i in mine))])
    dist.all_reduce(bodies)
    q.put((rank, shards, float(bodies.item()), sum(counts)))
    dist.barrier()
    dist.destroy_process_group()


def test_ensemble_instances_split_across_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_ensemble_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, shards, bodies, total in out:
        flat = sorted(i for sh in shards for i in sh)
        assert flat == list(range(64))                      # every instance exactly once
        assert len(shards[0]) == len(shards[1]) == 32
        assert bodies == total                               # the job's bodies are the ensemble's
