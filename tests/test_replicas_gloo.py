"""Multi-rank path of bench.py on CPU: two gloo ranks (127.0.0.1) each time an
independent replica; the job time is the max over ranks and the whole-job
throughput counts every replica's steps (replicas only: a single sheet does
not shard, so no collective touches the data path)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    ms = [100.0 + 50.0 * rank, 200.0 - 10.0 * rank]  # rank 1 is the slower replica in the first timing
    out = bench.max_over_ranks(ms, "cpu", world)
    q.put((rank, out, bench.replica_throughput(world, 20, out[0])))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_and_replica_throughput():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    res = sorted(q.get(timeout=5) for _ in range(world))
    for rank, out, thr in res:
        assert out == [150.0, 200.0]          # both ranks agree on the slowest replica
        assert thr == pytest.approx(2 * 20 / 0.150)
