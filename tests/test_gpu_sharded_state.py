"""One state over several ranks on the GPU: every rank's shard an engine
StateVector run by fused plans, the exchanges between segments by device
copies -- all ranks hosted in one process on one GPU (the ranks' kernels do
not wait on one another: each exchange is a set of copies between whole
launches).  Against the FP64 oracle."""
import numpy as np
import pytest

import oracle
from subquokka_dev_b200 import circuits
from subquokka_dev_b200.sharding import EngineShards, ShardedStateVector

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind,n,world,dtype,tol", [("random_u3_cz", 16, 2, "c128", 1e-12),
                                                    ("random_u3_cz", 16, 4, "c128", 1e-12),
                                                    ("qft", 15, 8, "c128", 1e-12),
                                                    ("hea", 14, 4, "c128", 1e-12),
                                                    ("random_u3_cz", 16, 4, "c64", 2e-6)])
def test_sharded_state_on_one_gpu_matches_oracle(kind, n, world, dtype, tol):
    circ = (circuits.random_u3_cz(n, 8, 31) if kind == "random_u3_cz" else circuits.qft(n) if kind == "qft"
            else circuits.hea(n, 4, 32)[0])
    sv = ShardedStateVector(n, world=world, ranks=range(world), backend=EngineShards(dtype))
    sv.apply(circ)
    out = sv.gather()
    sv.close()
    z = np.zeros(1 << n, np.complex128)
    z[0] = 1
    assert sv.exchanges >= 1
    assert np.abs(out - oracle.apply_circuit(z, n, circ)).max() <= tol


def test_sharded_state_per_gate_shards():
    n, world = 13, 2
    circ = circuits.random_u3_cz(n, 5, 33)
    sv = ShardedStateVector(n, world=world, ranks=range(world), backend=EngineShards("c128", fused=False))
    sv.apply(circ)
    out = sv.gather()
    sv.close()
    z = np.zeros(1 << n, np.complex128)
    z[0] = 1
    assert np.abs(out - oracle.apply_circuit(z, n, circ)).max() <= 1e-12
