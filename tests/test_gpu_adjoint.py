"""Expectation values and adjoint gradients on the GPU against the FP64
oracle: Pauli expectations, CPU parameter shift, central finite differences."""
import numpy as np
import pytest
import torch

import oracle
from subquokka_dev_b200 import StateVector, adjoint_grad, circuits, expval, make_gate, zz_x_hamiltonian
from subquokka_dev_b200.torch_shim import ParamCircuit, expectation, hea_template

pytestmark = pytest.mark.gpu


def random_terms(n, k, seed):
    rng = np.random.default_rng(seed)
    return [(float(rng.standard_normal()), int(rng.integers(1 << n)), int(rng.integers(1 << n))) for _ in range(k)]


@pytest.mark.parametrize("dtype,tol", [("c128", 1e-12), ("c64", 2e-5)])
def test_expval_pauli_sum(dtype, tol):
    n = 11
    s = circuits.random_state(n, 12)
    terms = random_terms(n, 40, 13) + zz_x_hamiltonian(n, np.ones(n - 1), np.ones(n))
    with StateVector(n, dtype) as sv:
        sv.upload(s)
        got = expval(sv, terms)
    assert abs(got - oracle.pauli_expval(s, n, terms)) <= tol


def hea_problem(n, layers, seed):
    pc = hea_template(n, layers)
    rng = np.random.default_rng(seed)
    params = rng.uniform(-np.pi, np.pi, pc.nparams)
    terms = zz_x_hamiltonian(n, rng.standard_normal(n - 1), rng.standard_normal(n))
    return pc, params, terms


@pytest.mark.parametrize("fused", [False, True])
@pytest.mark.parametrize("checkpoints", [0, 3, -1])
def test_adjoint_matches_parameter_shift_c128(checkpoints, fused):
    n, layers = 9, 3
    pc, params, terms = hea_problem(n, layers, 21)
    circ, idx = pc.bind(params)
    with StateVector(n) as sv:
        ev, grad, drift = adjoint_grad(sv, circ, idx, pc.nparams, terms, checkpoints, fused)
        back = sv.download()
    ps = oracle.param_shift_grad(pc, params, terms)
    z0 = np.zeros(1 << n, complex)
    z0[0] = 1
    assert abs(ev - oracle.pauli_expval(oracle.apply_circuit(z0, n, circ), n, terms)) < 1e-12
    assert np.abs(grad - ps).max() <= 1e-10 * max(1.0, np.abs(ps).max())
    assert drift < 1e-12
    assert np.abs(back - z0).max() < 1e-12   # the sweep uncomputes back to |0>


@pytest.mark.parametrize("fused", [False, True])
def test_adjoint_c64_close_to_fp64(fused):
    n, layers = 10, 3
    pc, params, terms = hea_problem(n, layers, 22)
    circ, idx = pc.bind(params)
    with StateVector(n, "c64") as sv:
        ev, grad, drift = adjoint_grad(sv, circ, idx, pc.nparams, terms, -1, fused)
    ps = oracle.param_shift_grad(pc, params, terms)
    assert np.abs(grad - ps).max() <= 1e-4 * np.abs(ps).max()
    assert drift < 1e-4


@pytest.mark.parametrize("fused", [False, True])
def test_shared_parameters_and_fixed_gates(fused):
    # one parameter on several gates, RX included, non-trainable gates of every kind
    n = 7
    pc = ParamCircuit(n)
    a, b = pc.param(), pc.param()
    for q in range(n):
        pc.fixed("H", [q])
        pc.rot("RX", q, a)
        pc.rot("RZ", q, b)
    pc.fixed("CP", [0, 3], 0.7)
    pc.fixed("RZZ", [2, 5], 0.3)
    pc.fixed("SWAP", [1, 6])
    pc.u3(4, a, b, a)
    pc.fixed("VSWAP", [0, 1, 5, 6])
    params = np.array([0.4, -1.1])
    terms = random_terms(n, 10, 23)
    circ, idx = pc.bind(params)
    with StateVector(n) as sv:
        _, grad, _ = adjoint_grad(sv, circ, idx, pc.nparams, terms, -1, fused)
    assert np.abs(grad - oracle.param_shift_grad(pc, params, terms)).max() < 1e-10


def test_torch_shim_backward():
    n, layers = 8, 2
    pc, params, terms = hea_problem(n, layers, 24)
    p = torch.tensor(params, dtype=torch.float64, requires_grad=True)
    e = expectation(p, pc, terms)
    e.backward()
    assert np.abs(p.grad.numpy() - oracle.param_shift_grad(pc, params, terms)).max() < 1e-10


@pytest.mark.parametrize("fused", [False, True])
def test_adjoint_vs_central_differences_larger_state(fused):
    # 20 qubits: a few parameters checked by central differences on the GPU
    n, layers = 20, 2
    pc, params, terms = hea_problem(n, layers, 25)
    circ, idx = pc.bind(params)
    with StateVector(n) as sv:
        _, grad, drift = adjoint_grad(sv, circ, idx, pc.nparams, terms, -1, fused)
    eps = 1e-5
    for p in (0, 7, pc.nparams // 2, pc.nparams - 1):
        e = []
        for sg in (1, -1):
            v = params.copy()
            v[p] += sg * eps
            c2, _ = pc.bind(v)
            with StateVector(n) as sv:
                sv.apply(c2)
                e.append(expval(sv, terms))
        fd = (e[0] - e[1]) / (2 * eps)
        assert abs(fd - grad[p]) <= 1e-6 * max(1.0, abs(grad[p]))


def test_fused_and_per_gate_adjoint_agree_at_scale():
    n, layers = 22, 4
    pc, params, terms = hea_problem(n, layers, 26)
    circ, idx = pc.bind(params)
    out = []
    for fused in (False, True):
        with StateVector(n) as sv:
            out.append(adjoint_grad(sv, circ, idx, pc.nparams, terms, -1, fused))
    assert abs(out[0][0] - out[1][0]) < 1e-12
    assert np.abs(out[0][1] - out[1][1]).max() < 1e-11


@pytest.mark.parametrize("fused", [False, True])
def test_adjoint_matches_c_restatement(fused):
    n, layers = 12, 4
    pc, params, terms = hea_problem(n, layers, 27)
    circ, idx = pc.bind(params)
    z0 = np.zeros(1 << n, complex)
    z0[0] = 1
    ev0, g0 = oracle.adjoint_grad(z0, n, circ, idx, pc.nparams, terms)
    with StateVector(n) as sv:
        ev, g, _ = adjoint_grad(sv, circ, idx, pc.nparams, terms, -1, fused)
    assert abs(ev - ev0) < 1e-12
    assert np.abs(g - g0).max() < 1e-11


@pytest.mark.parametrize("fused", [False, True])
def test_workspace_reuse_and_release(fused):
    # the lambda / checkpoint workspace stays with the state between calls,
    # grows when a call needs more checkpoints, and can be released; results
    # do not depend on its history
    n, layers = 11, 4
    pc, params, terms = hea_problem(n, layers, 28)
    circ, idx = pc.bind(params)
    with StateVector(n) as sv:
        ref = adjoint_grad(sv, circ, idx, pc.nparams, terms, 0, fused)
        runs = [adjoint_grad(sv, circ, idx, pc.nparams, terms, c, fused) for c in (0, 5, 2, 0)]
        z0 = np.zeros(1 << n, complex)
        z0[0] = 1
        assert abs(expval(sv, terms) - oracle.pauli_expval(z0, n, terms)) < 1e-12   # shares the accumulator
        sv.release_workspace()
        runs.append(adjoint_grad(sv, circ, idx, pc.nparams, terms, 3, fused))
        sv.release_workspace()
        sv.release_workspace()
    for ev, g, drift in runs:
        assert abs(ev - ref[0]) < 1e-12
        assert np.abs(g - ref[1]).max() < 1e-11
        assert drift < 1e-12


def test_last_sweep_reports_device_time_and_traffic():
    """qk_sv_last_sweep: CUDA-event time of the sweep and, for the fused form,
    its algorithmic bytes = 2S per forward pass + 4S per two-state pass + the
    H application, reductions and checkpoint copies."""
    from subquokka_dev_b200 import QkError, last_sweep
    n = 14
    pc = hea_template(n, 3)
    rng = np.random.default_rng(5)
    params = rng.uniform(-np.pi, np.pi, pc.nparams)
    terms = zz_x_hamiltonian(n, rng.standard_normal(n - 1), rng.standard_normal(n))
    circ, idx = pc.bind(params)
    with StateVector(n, "c64") as sv:
        with pytest.raises(QkError):
            last_sweep(sv)                       # nothing has run yet
        adjoint_grad(sv, circ, idx, pc.nparams, terms, 0, True)
        st = last_sweep(sv)
        S = 8 << n
        assert st["device_ms"] > 0 and st["forward_passes"] > 0 and st["backward_passes"] > 0
        assert st["alg_bytes"] >= 2 * S * st["forward_passes"] + 4 * S * st["backward_passes"]
        adjoint_grad(sv, circ, idx, pc.nparams, terms, 0, False)
        st = last_sweep(sv)
        assert st["alg_bytes"] == 0 and st["forward_passes"] == circ.ngates
