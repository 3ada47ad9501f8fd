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


# ---- batch sharding: the partition and the one collective that gathers results

def test_partition_covers_every_circuit_once_and_balances_cost():
    import numpy as np
    from subquokka_dev_b200 import circuits
    from subquokka_dev_b200.sharding import circuit_cost, partition
    items = circuits.variational_batch(256, 2025)
    costs = [circuit_cost(pc) for pc, _, _ in items]
    for world in (1, 2, 3, 4, 8):
        parts = partition(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(256))
        loads = [sum(costs[i] for i in p) for p in parts]
        # LPT bound: the heaviest rank exceeds the mean by at most one circuit's cost
        assert max(loads) - sum(loads) / world <= max(costs) + 1e-9
        assert partition(costs, world) == parts          # every rank computes the same split


def _sharded_worker(rank, world, port, out):
    import datetime
    import numpy as np
    import torch.distributed as dist
    from subquokka_dev_b200.sharding import gather_results, partition
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    pcounts = [3, 5, 2, 7, 1, 4]
    costs = [8.0, 1.0, 6.0, 2.0, 5.0, 3.0]
    mine = partition(costs, world)[rank]
    # stand-in results of circuit c: <H> = c + 0.5, drift = -c, gradient = c * 10 + arange
    local = (np.array([c + 0.5 for c in mine]), [c * 10 + np.arange(pcounts[c], dtype=float) for c in mine],
             np.array([-float(c) for c in mine]))
    ev, grads, drift = gather_results(mine, local, pcounts, "cpu")
    out.put((rank, mine, ev.tolist(), [g.tolist() for g in grads], drift.tolist()))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_gather_a_sharded_batch():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_sharded_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    pcounts = [3, 5, 2, 7, 1, 4]
    assert sorted(res[0][1] + res[1][1]) == list(range(6)) and res[0][1] and res[1][1]
    for rank, mine, ev, grads, drift in res:
        assert ev == [c + 0.5 for c in range(6)]
        assert drift == [-float(c) for c in range(6)]
        assert grads == [[c * 10 + k for k in range(pcounts[c])] for c in range(6)]
