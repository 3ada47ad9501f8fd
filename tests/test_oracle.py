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


def test_pauli_expval_matches_dense_operators():
    n = 5
    s = circuits.random_state(n, 9)
    rng = np.random.default_rng(3)
    I, X = np.eye(2), np.array([[0, 1], [1, 0]], dtype=complex)
    Y, Z = np.array([[0, -1j], [1j, 0]]), np.diag([1.0, -1.0]).astype(complex)
    terms, H = [], np.zeros((1 << n, 1 << n), complex)
    for _ in range(12):
        x, z = int(rng.integers(1 << n)), int(rng.integers(1 << n))
        c = float(rng.standard_normal())
        terms.append((c, x, z))
        op = np.array([[1.0 + 0j]])
        for q in reversed(range(n)):
            bx, bz = (x >> q) & 1, (z >> q) & 1
            op = np.kron(op, {(0, 0): I, (1, 0): X, (0, 1): Z, (1, 1): Y}[(bx, bz)])
        H += c * op
    assert abs(oracle.pauli_expval(s, n, terms) - np.vdot(s, H @ s).real) < 1e-12
    J, h = rng.standard_normal(n - 1), rng.standard_normal(n)
    from subquokka_dev_b200 import zz_x_hamiltonian
    assert abs(oracle.pauli_expval(s, n, zz_x_hamiltonian(n, J, h)) - oracle.expval_zz_x(s, n, J, h)) < 1e-12


def test_parameter_shift_matches_finite_differences():
    from subquokka_dev_b200 import zz_x_hamiltonian
    from subquokka_dev_b200.torch_shim import hea_template
    n, layers = 5, 2
    pc = hea_template(n, layers)
    rng = np.random.default_rng(4)
    params = rng.uniform(-np.pi, np.pi, pc.nparams)
    terms = zz_x_hamiltonian(n, rng.standard_normal(n - 1), rng.standard_normal(n))
    ps = oracle.param_shift_grad(pc, params, terms)
    z0 = np.zeros(1 << n, complex)
    z0[0] = 1
    eps = 1e-6
    for p in range(pc.nparams):
        e = []
        for sg in (1, -1):
            v = params.copy()
            v[p] += sg * eps
            e.append(oracle.pauli_expval(oracle.apply_circuit(z0, n, pc.bind(v)[0]), n, terms))
        assert abs((e[0] - e[1]) / (2 * eps) - ps[p]) < 1e-7


def test_c_adjoint_restatement_matches_parameter_shift():
    from subquokka_dev_b200 import zz_x_hamiltonian
    from subquokka_dev_b200.torch_shim import hea_template
    n, layers = 6, 3
    pc = hea_template(n, layers)
    rng = np.random.default_rng(8)
    params = rng.uniform(-np.pi, np.pi, pc.nparams)
    terms = zz_x_hamiltonian(n, rng.standard_normal(n - 1), rng.standard_normal(n)) + [(0.3, 0b101, 0b110)]
    circ, idx = pc.bind(params)
    z0 = np.zeros(1 << n, complex)
    z0[0] = 1
    ev, g = oracle.adjoint_grad(z0, n, circ, idx, pc.nparams, terms)
    assert abs(ev - oracle.pauli_expval(oracle.apply_circuit(z0, n, circ), n, terms)) < 1e-12
    assert np.abs(g - oracle.param_shift_grad(pc, params, terms)).max() < 1e-11
