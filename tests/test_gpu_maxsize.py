"""Largest states one B200 holds: 2^33 complex128 and 2^34 complex64
amplitudes (128 GiB each).  Every kernel class runs once with qubits at both
ends of the index, and the result is checked through Pauli expectation values
with closed forms (a host copy of 128 GiB is not made).  A wrong 64-bit index
anywhere shows up as an O(1) error."""
import numpy as np
import pytest

from subquokka_dev_b200 import Circuit, Plan, StateVector, expval, make_gate

pytestmark = pytest.mark.gpu

TH, PHI, LAM, PSI, A, B = 0.7, 1.1, 0.4, 0.9, 0.3, 1.3


def ry(t):
    return np.array([[np.cos(t / 2), -np.sin(t / 2)], [np.sin(t / 2), np.cos(t / 2)]], dtype=complex)


def circuit_and_expectations(n):
    top = n - 1
    cnot = np.eye(4)[[0, 1, 3, 2]]          # control = first (most significant) target
    g = [make_gate("H", [0]), make_gate("H", [top]), make_gate("CP", [0, top], np.pi),      # CZ |++>
         make_gate("RY", [3], TH), make_gate("RX", [n - 2], PHI),
         make_gate("H", [5]), make_gate("U2", [5, n - 3], coeff=cnot),                        # Bell pair
         make_gate("X", [4]), make_gate("SWAP", [4, n - 4]),
         make_gate("H", [1]), make_gate("RZZ", [1, n - 5], PSI),
         make_gate("H", [2]), make_gate("RZ", [2], LAM),
         make_gate("X", [6]), make_gate("VSWAP", [6, 7, n - 7, n - 6]),
         make_gate("U2", [8, 9], coeff=np.kron(ry(A), ry(B))),
         make_gate("H", [10]), make_gate("P", [10], np.pi / 2)]

    def z(*qs):
        return (0, sum(1 << q for q in qs))

    def x(*qs):
        return (sum(1 << q for q in qs), 0)

    def y(q):
        return (1 << q, 1 << q)

    expect = [(z(3), np.cos(TH)), (x(3), np.sin(TH)), (z(n - 2), np.cos(PHI)), (y(n - 2), -np.sin(PHI)),
              ((1 << 0, 1 << top), 1.0), (x(0), 0.0),
              (z(5, n - 3), 1.0), (x(5, n - 3), 1.0), (z(5), 0.0),
              (z(4), 1.0), (z(n - 4), -1.0),
              (x(1), np.cos(PSI)), (y(1), np.sin(PSI)), (x(2), np.cos(LAM)), (y(2), np.sin(LAM)),
              (z(6), 1.0), (z(n - 7), -1.0), (z(7), 1.0), (z(n - 6), 1.0),
              (z(8), np.cos(A)), (z(9), np.cos(B)), (y(10), 1.0), (x(10), 0.0)]
    return Circuit(g), expect


@pytest.mark.parametrize("n,dtype,forms,tol", [
    (33, "c128", ("per_gate", "passes", "tensor_cores"), 1e-9),   # the H literal 0.70710678118 loses ~1e-11 a gate
    (34, "c64", ("per_gate", "passes", "tensor_cores"), 2e-5),
])
def test_largest_state(n, dtype, forms, tol):
    import torch
    torch.cuda.empty_cache()   # device memory cached by earlier tests' tensors
    circ, expect = circuit_and_expectations(n)
    with StateVector(n, dtype) as sv:
        for form in forms:
            sv.reset()
            if form == "per_gate":
                sv.apply(circ)
            else:
                plan = Plan(circ, n, dtype, fuse_width=6 if form == "tensor_cores" else 0)
                plan.apply(sv)
                plan.close()
            for (xm, zm), want in expect:
                coeff = 1.0
                got = expval(sv, [(coeff, xm, zm)])
                assert abs(got - want) <= tol, (form, hex(xm), hex(zm), got, want)
