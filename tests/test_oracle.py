"""The oracle (C restatement of the reference's MEM gates) pinned against the
golden states the unmodified reference produced, plus analytic known answers."""
import numpy as np
import pytest

import oracle
from subquokka_dev_b200 import Circuit, circuits, make_gate

import golden_util as gu


@pytest.mark.parametrize("name", gu.names())
def test_oracle_matches_reference_golden(name):
    rec = gu.load(name)
    n = rec["n"]
    circ = Circuit.parse(rec["circuit"], rec["is_subcircuit"], n)
    final = oracle.apply_circuit(gu.initial_state(rec), n, circ)
    assert gu.compare(rec, final) <= 1e-12


def test_hadamard_all_qubits_known_answer():
    # every amplitude of H^n |0> is 0.70710678118^n (the reference's literal,
    # src/circuit.cpp:245-248)
    n = 9
    s = np.zeros(1 << n, np.complex128)
    s[0] = 1
    out = oracle.apply_circuit(s, n, Circuit([make_gate("H", [q]) for q in range(n)]))
    assert np.allclose(out, 0.70710678118 ** n, rtol=0, atol=1e-15)


def test_rx_pi_all_qubits_known_answer():
    # RX(pi)^n |0> = (-i)^n |1...1> (the reference's rxN.txt benchmark circuits)
    n = 7
    s = np.zeros(1 << n, np.complex128)
    s[0] = 1
    out = oracle.apply_circuit(s, n, Circuit([make_gate("RX", [q], np.pi) for q in range(n)]))
    exp = np.zeros_like(s)
    exp[-1] = (-1j) ** n
    assert np.abs(out - exp).max() < 1e-12


def test_qft_of_zero_is_uniform():
    n = 8
    s = np.zeros(1 << n, np.complex128)
    s[0] = 1
    out = oracle.apply_circuit(s, n, circuits.qft(n))
    assert np.allclose(out, 0.70710678118 ** n, atol=1e-12)


def test_expval_matches_dense_numpy():
    n = 6
    s = circuits.random_state(n, 5)
    rng = np.random.default_rng(1)
    J, h = rng.standard_normal(n - 1), rng.standard_normal(n)
    Z = np.diag([1.0, -1.0])
    X = np.array([[0.0, 1.0], [1.0, 0.0]])

    def op(mats):
        out = np.array([[1.0]])
        for q in reversed(range(n)):
            out = np.kron(out, mats.get(q, np.eye(2)))
        return out
    H = sum(J[i] * op({i: Z, i + 1: Z}) for i in range(n - 1)) + sum(h[i] * op({i: X}) for i in range(n))
    assert abs(oracle.expval_zz_x(s, n, J, h) - np.vdot(s, H @ s).real) < 1e-12
