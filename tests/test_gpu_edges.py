"""Edge cases on the GPU against the FP64 oracle: tiny states, empty gate
lists, and U2 matrices that run as a cheaper op (CNOT either way round, SWAP,
diagonal)."""
import numpy as np
import pytest

import oracle
from subquokka_dev_b200 import Circuit, Plan, StateVector, adjoint_grad, circuits, expval, make_gate, zz_x_hamiltonian

pytestmark = pytest.mark.gpu

KINDS1 = ["H", "X", "Y", "Z", "P", "RX", "RY", "RZ", "U1"]


def random_gates(n, count, seed):
    rng = np.random.default_rng(seed)
    gates = []
    for _ in range(count):
        if n > 1 and rng.random() < 0.4:
            a, b = sorted(int(x) for x in rng.choice(n, 2, replace=False))
            k = ["CP", "RZZ", "SWAP", "U2"][rng.integers(4)]
            if k == "U2":
                z = rng.standard_normal((4, 4)) + 1j * rng.standard_normal((4, 4))
                gates.append(make_gate(k, [a, b], coeff=np.linalg.qr(z)[0]))
            elif k == "SWAP":
                gates.append(make_gate(k, [a, b]))
            else:
                gates.append(make_gate(k, [a, b], rng.uniform(-4, 4)))
        else:
            k = KINDS1[rng.integers(len(KINDS1))]
            q = [int(rng.integers(n))]
            if k == "U1":
                z = rng.standard_normal((2, 2)) + 1j * rng.standard_normal((2, 2))
                gates.append(make_gate(k, q, coeff=np.linalg.qr(z)[0]))
            elif k in ("P", "RX", "RY", "RZ"):
                gates.append(make_gate(k, q, rng.uniform(-4, 4)))
            else:
                gates.append(make_gate(k, q))
    return Circuit(gates)


@pytest.mark.parametrize("n", [1, 2, 3, 5])
def test_tiny_states_every_path(n):
    circ = random_gates(n, 40, 100 + n)
    init = circuits.random_state(n, 101)
    ref = oracle.apply_circuit(init, n, circ)
    for dtype, tol in (("c128", 1e-12), ("c64", 2e-6)):
        with StateVector(n, dtype) as sv:
            sv.upload(init)
            sv.apply(circ)
            assert np.abs(sv.download() - ref).max() <= tol, ("per-gate", dtype)
            sv.upload(init)
            with sv.capture(circ) as g:
                g.launch()
            assert np.abs(sv.download() - ref).max() <= tol, ("graph", dtype)
            sv.upload(init)
            p = Plan(circ, n, dtype)
            p.apply(sv)
            p.close()
            assert np.abs(sv.download() - ref).max() <= tol, ("fused", dtype)


def test_empty_gate_lists():
    n = 6
    init = circuits.random_state(n, 102)
    empty = Circuit([])
    terms = zz_x_hamiltonian(n, np.ones(n - 1), np.ones(n))
    with StateVector(n) as sv:
        sv.upload(init)
        sv.apply(empty)
        with sv.capture(empty) as g:
            g.launch()
        p = Plan(empty, n)
        p.apply(sv)
        p.close()
        assert np.array_equal(sv.download(), init)
        ev = expval(sv, terms)
        for fused in (False, True):
            e2, grad, drift = adjoint_grad(sv, empty, np.zeros(0, np.int32), 0, terms, -1, fused)
            assert abs(e2 - ev) < 1e-12 and grad.size == 0 and drift == 0
        assert np.abs(sv.download() - init).max() < 1e-15
    assert abs(ev - oracle.pauli_expval(init, n, terms)) < 1e-12


CNOT_BE = np.array([[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 0, 1], [0, 0, 1, 0]], dtype=complex)   # control = first qubit
CNOT_BE_REV = np.array([[1, 0, 0, 0], [0, 0, 0, 1], [0, 0, 1, 0], [0, 1, 0, 0]], dtype=complex)
SWAP_M = np.array([[1, 0, 0, 0], [0, 0, 1, 0], [0, 1, 0, 0], [0, 0, 0, 1]], dtype=complex)
DIAG_M = np.diag(np.exp(1j * np.array([0.3, -1.1, 2.0, 0.7])))
PHASED_PERM = np.array([[0, 1j, 0, 0], [1, 0, 0, 0], [0, 0, 0, -1], [0, 0, 1, 0]], dtype=complex)  # stays dense


@pytest.mark.parametrize("mat", [CNOT_BE, CNOT_BE_REV, SWAP_M, DIAG_M, PHASED_PERM],
                         ids=["cnot", "cnot_reversed", "swap", "diagonal", "phased_permutation"])
def test_structured_u2_matrices(mat):
    # U2 in the reference's big-endian coefficient order on many qubit pairs:
    # per-gate, fused c128 and tensor-core c64 paths against the oracle's
    # dense 4 x 4 product
    n = 13
    init = circuits.random_state(n, 103)
    pairs = [(0, 1), (0, 7), (2, 3), (3, 12), (6, 11), (11, 12)]
    circ = Circuit([make_gate("U2", [a, b], coeff=mat) for a, b in pairs] +
                   [make_gate("H", [q]) for q in range(n)] +
                   [make_gate("U2", [a, b], coeff=mat) for a, b in reversed(pairs)])
    ref = oracle.apply_circuit(init, n, circ)
    with StateVector(n) as sv:
        sv.upload(init)
        sv.apply(circ)
        assert np.abs(sv.download() - ref).max() <= 1e-12
        sv.upload(init)
        p = Plan(circ, n)
        p.apply(sv)
        p.close()
        assert np.abs(sv.download() - ref).max() <= 1e-12
    with StateVector(n, "c64") as sv:
        sv.upload(init)
        p = Plan(circ, n, "c64", fuse_width=6)
        p.apply(sv)
        p.close()
        assert np.abs(sv.download() - ref).max() <= 5e-5
