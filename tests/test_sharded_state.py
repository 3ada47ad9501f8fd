"""One state over several ranks (global-qubit sharding), on the CPU: the
exchange logic (which qubits move, where blocks go, how positions are
tracked) with every rank's shard a numpy array and its local gates applied by
the FP64 oracle -- all ranks in one process, and two / four gloo ranks with
the all-to-all as the only exchange.  The GPU runs of the same class are in
tests/test_gpu_sharded_state.py."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

import oracle
from subquokka_dev_b200 import circuits
from subquokka_dev_b200.sharding import ShardedStateVector


class OracleShards:
    """Test backend: a shard is a complex128 numpy array (as a torch view),
    gate lists applied by the CPU oracle."""

    def zero(self, m, first):
        a = np.zeros(1 << m, np.complex128)
        if first:
            a[0] = 1
        return {"cur": a, "other": np.zeros(1 << m, np.complex128), "m": m}

    def tensor(self, sh):
        return torch.from_numpy(sh["cur"])

    def scratch(self, sh):
        return torch.from_numpy(sh["other"])

    def swap_in(self, sh):
        sh["cur"], sh["other"] = sh["other"], sh["cur"]

    def apply(self, sh, circ, m):
        if circ.ngates:
            sh["cur"][:] = oracle.apply_circuit(sh["cur"], m, circ)

    def close(self, sh):
        pass


CASES = [("random_u3_cz", 10, 2), ("random_u3_cz", 10, 4), ("qft", 9, 4), ("qft", 10, 8), ("hea", 9, 2),
         ("mixed", 9, 4)]


def build(kind, n):
    if kind == "random_u3_cz":
        return circuits.random_u3_cz(n, 6, 17)
    if kind == "qft":
        return circuits.qft(n)
    if kind == "mixed":   # H, RX, CP, RZZ, SWAP, VSWAP_2_2 on random qubits
        from test_ooc_host import random_mixed
        return random_mixed(n, 150, 19)
    return circuits.hea(n, 3, 18)[0]


@pytest.mark.parametrize("kind,n,world", CASES)
def test_all_ranks_in_one_process_match_the_oracle(kind, n, world):
    circ = build(kind, n)
    sv = ShardedStateVector(n, world=world, ranks=range(world), backend=OracleShards())
    sv.apply(circ)
    z = np.zeros(1 << n, np.complex128)
    z[0] = 1
    assert np.abs(sv.gather() - oracle.apply_circuit(z, n, circ)).max() <= 1e-12
    assert sv.exchanges >= 1   # the circuits touch every qubit: global ones had to move


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, n, out):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    circ = circuits.random_u3_cz(n, 5, 23)
    sv = ShardedStateVector(n, backend=OracleShards())
    sv.apply(circ)
    full = sv.gather()
    out.put((rank, sv.exchanges, full if rank == 0 else None))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 4])
def test_gloo_ranks_exchange_by_all_to_all(world):
    n = 9
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, n, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=180) for _ in procs), key=lambda x: x[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert len({x[1] for x in res}) == 1          # every rank took the same exchanges
    z = np.zeros(1 << n, np.complex128)
    z[0] = 1
    ref = oracle.apply_circuit(z, n, circuits.random_u3_cz(n, 5, 23))
    assert np.abs(res[0][2] - ref).max() <= 1e-12
