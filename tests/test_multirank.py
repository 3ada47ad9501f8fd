"""The N > 1 path of bench.py (independent replicas, one per rank) on CPU with
two gloo ranks: the only collective is the max of the per-rank times."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    local_ms = 100.0 + 50.0 * rank            # rank 1 is the slow replica
    m = bench.max_over_ranks(local_ms, world, device="cpu")
    v = bench.replica_throughput(world, 10**9, 2, m)
    out.put((rank, m, v))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_aggregate_replicas():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, m, v in res:
        assert m == 150.0                        # both ranks see the slowest time
        assert v == pytest.approx(2 * 1e9 * 2 / 0.150 / 1e9)


def test_single_rank_needs_no_collective():
    import bench
    assert bench.max_over_ranks(3.5, 1) == 3.5
