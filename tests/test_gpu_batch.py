"""Batched variational circuits (one CUDA graph, one persistent launch per
step) against the single-circuit adjoint path and the FP64 oracle."""
import numpy as np
import pytest

import oracle
from subquokka_dev_b200 import Batch, StateVector, adjoint_grad, circuits

pytestmark = pytest.mark.gpu


def single(pc, params, terms, dtype):
    circ, idx = pc.bind(params)
    with StateVector(pc.n, dtype) as sv:
        ev, g, _ = adjoint_grad(sv, circ, idx, pc.nparams, terms, 0, False)
    return ev, g


@pytest.mark.parametrize("dtype,tol", [("c128", 1e-11), ("c64", 2e-4)])
def test_batch_matches_single_circuits(dtype, tol):
    items = circuits.variational_batch(7, 50, qmin=9, qmax=15, lmin=1, lmax=5)
    b = Batch(items, dtype)
    ev, grads, drift = b.run()
    for c, (pc, params, terms) in enumerate(items):
        e1, g1 = single(pc, params, terms, "c128")
        assert abs(ev[c] - e1) <= tol * max(1, abs(e1)), c
        assert np.abs(grads[c] - g1).max() <= tol * max(1, np.abs(g1).max()), c
    assert drift.max() < (1e-10 if dtype == "c128" else 1e-4)
    st = b.stats()
    assert st["steps"] >= 2 and st["launches"] == st["steps"] + 3
    b.close()


def test_batch_against_parameter_shift():
    items = circuits.variational_batch(3, 51, qmin=5, qmax=7, lmin=1, lmax=3)
    b = Batch(items, "c128")
    ev, grads, _ = b.run()
    for c, (pc, params, terms) in enumerate(items):
        assert np.abs(grads[c] - oracle.param_shift_grad(pc, params, terms)).max() < 1e-10
    b.close()


def test_batch_set_params_and_rerun():
    items = circuits.variational_batch(4, 52, qmin=10, qmax=13, lmin=2, lmax=4)
    b = Batch(items, "c128")
    b.run()
    rng = np.random.default_rng(9)
    new = [rng.uniform(-3, 3, pc.nparams) for pc, _, _ in items]
    b.set_params(new)
    ev, grads, _ = b.run()
    for c, (pc, _, terms) in enumerate(items):
        e1, g1 = single(pc, new[c], terms, "c128")
        assert abs(ev[c] - e1) < 1e-11 and np.abs(grads[c] - g1).max() < 1e-11
    b.close()


@pytest.mark.parametrize("dtype,tol", [("c64", 2e-4), ("c128", 1e-11)])
def test_batch_autotune_gives_same_results(dtype, tol):
    # every candidate tile shape (complex128: 16 register amplitudes a thread
    # included) gives the default shape's results
    items = circuits.variational_batch(5, 53, qmin=13, qmax=16, lmin=2, lmax=4)
    ref = Batch(items, dtype)
    auto = Batch(items, dtype, autotune=True)
    e0, g0, _ = ref.run()
    e1, g1, _ = auto.run()
    assert np.abs(e0 - e1).max() < tol
    for a, c in zip(g0, g1):
        assert np.abs(a - c).max() < tol * max(1, np.abs(a).max())
    ref.close()
    auto.close()


def test_sharded_batch_shards_give_the_whole_batch():
    """The shards of a ShardedBatch (here all ranks of a 3-way split run in
    this one process, one after another, on one GPU) reassemble into the
    unsharded batch's results: the partition and the result layout lose
    nothing."""
    from subquokka_dev_b200.sharding import ShardedBatch
    items = circuits.variational_batch(9, 52, qmin=8, qmax=13, lmin=1, lmax=4)
    whole = Batch(items, "c128")
    ev, grads, drift = whole.run()
    whole.close()
    got_ev = np.full(len(items), np.nan)
    got_g = [None] * len(items)
    for rank in range(3):
        sb = ShardedBatch(items, "c128", rank=rank, world=3)
        e, g, d = sb.run()      # no process group: this rank's circuits, zeros elsewhere
        for c in sb.mine:
            got_ev[c], got_g[c] = e[c], g[c]
        assert sb.device_ms() > 0
        sb.close()
    assert np.abs(got_ev - ev).max() <= 1e-12
    for c in range(len(items)):
        assert np.abs(got_g[c] - grads[c]).max() <= 1e-12


def test_batch_timing_reports_device_time_and_bytes():
    items = circuits.variational_batch(4, 53, qmin=8, qmax=10, lmin=1, lmax=2)
    b = Batch(items, "c64")
    b.run()
    ms, nbytes = b.timing()
    # at least a forward and a backward pass, reset, H and drift per circuit
    assert ms > 0 and nbytes >= sum(10 * (8 << pc.n) for pc, _, _ in items)
    b.close()
