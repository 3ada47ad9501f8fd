"""Seeded synthetic circuits in the reference's circuit.txt grammar.

These are the benchmark and test workloads.  Each one is written with the
gate tokens the reference's MEM parser accepts (src/simulator.cpp:542-597):
a single-qubit U3(theta, phi, lambda) becomes ``U1 q`` with its 2x2 matrix, CZ
becomes ``CP a b pi`` and CNOT becomes ``U2 c t`` with the CNOT matrix in the
reference's big-endian U2 order (src/circuit.cpp:2807-2819).
"""
from __future__ import annotations

import math

import numpy as np

from .engine import Circuit, make_gate


def qft(n: int) -> Circuit:
    """QFT as generated by the reference's python_script/cir_qft.py:27-35:
    for i: H i; CP i j pi/2^(j-i) for j > i; then SWAP i n-1-i."""
    gates = []
    for i in range(n):
        gates.append(make_gate("H", [i]))
        angle = math.pi / 2
        for j in range(i + 1, n):
            gates.append(make_gate("CP", [i, j], angle))
            angle /= 2
    for i in range(n // 2):
        gates.append(make_gate("SWAP", [i, n - 1 - i]))
    return Circuit(gates)


def u3_matrix(theta: float, phi: float, lam: float) -> np.ndarray:
    c, s = math.cos(theta / 2), math.sin(theta / 2)
    return np.array([[c, -np.exp(1j * lam) * s],
                     [np.exp(1j * phi) * s, np.exp(1j * (phi + lam)) * c]], dtype=np.complex128)


def random_u3_cz(n: int, layers: int, seed: int) -> Circuit:
    """Random circuit: per layer a U3 on every qubit (angles uniform in
    [0, 2 pi) drawn in (layer, qubit, theta/phi/lambda) order), then CZ on the
    brick pairs (0,1),(2,3),... in even layers and (1,2),(3,4),... in odd ones."""
    rng = np.random.default_rng(seed)
    ang = rng.uniform(0.0, 2 * math.pi, size=(layers, n, 3))
    gates = []
    for l in range(layers):
        for q in range(n):
            gates.append(make_gate("U1", [q], coeff=u3_matrix(*ang[l, q])))
        for a in range(l % 2, n - 1, 2):
            gates.append(make_gate("CP", [a, a + 1], math.pi))
    return Circuit(gates)


CNOT_BIG_ENDIAN = np.array([[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 0, 1], [0, 0, 1, 0]], dtype=np.complex128)


def hea(n: int, layers: int, seed: int):
    """Hardware-efficient ansatz: per layer RY(theta) and RZ(phi) on every
    qubit, then a CNOT ladder i -> i+1.  Parameters uniform in [-pi, pi).
    Returns (circuit, params, J, h) with J, h ~ N(0, 1) for
    H = sum_i J_i Z_i Z_{i+1} + sum_i h_i X_i."""
    rng = np.random.default_rng(seed)
    params = rng.uniform(-math.pi, math.pi, size=(layers, n, 2))
    J = rng.standard_normal(n - 1)
    h = rng.standard_normal(n)
    gates = []
    for l in range(layers):
        for q in range(n):
            gates.append(make_gate("RY", [q], params[l, q, 0]))
            gates.append(make_gate("RZ", [q], params[l, q, 1]))
        for q in range(n - 1):
            gates.append(make_gate("U2", [q, q + 1], coeff=CNOT_BIG_ENDIAN))
    return Circuit(gates), params.ravel(), J, h


def random_state(n: int, seed: int) -> np.ndarray:
    """Seeded random normalised complex128 state: re, im i.i.d. N(0, 1)."""
    rng = np.random.default_rng(seed)
    a = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    return (a / np.linalg.norm(a)).astype(np.complex128)


def algorithmic_bytes(circuit: Circuit, n: int, amp_bytes: int = 16) -> int:
    """Bytes each gate must read and write: dense 2S, one-qubit diagonal S
    (Z, P) or 2S (RZ), CP S/2, SWAP S, VSWAP_k_k (1 - 2^-k) 2S, with S the
    state size."""
    S = amp_bytes << n
    total = 0
    for g in circuit.gate_list():
        name = {1: "H", 2: "X", 3: "Y", 4: "Z", 5: "P", 6: "RX", 7: "RY", 8: "RZ", 9: "U1", 10: "U2",
                11: "SWAP", 12: "CP", 13: "RZZ", 14: "VSWAP", 15: "MPI_VSWAP"}[g.kind]
        if name in ("Z", "P"):
            total += S
        elif name == "CP":
            total += S // 2
        elif name in ("SWAP",) or (name in ("VSWAP", "MPI_VSWAP") and g.nq == 2):
            total += S
        elif name in ("VSWAP", "MPI_VSWAP"):
            k = g.nq // 2
            total += int(2 * S * (1 - 2.0 ** -k))
        else:
            total += 2 * S
    return total


def variational_batch(ncirc: int, seed: int, qmin: int = 14, qmax: int = 22, lmin: int = 4, lmax: int = 16):
    """Batch of hardware-efficient-ansatz circuits of uneven size: qubits
    uniform in [qmin, qmax], layers uniform in [lmin, lmax], parameters uniform
    in [-pi, pi), per-circuit H = sum J_i Z_i Z_{i+1} + sum h_i X_i with J, h
    ~ N(0, 1).  Returns [(ParamCircuit, params, terms), ...]."""
    from .engine import zz_x_hamiltonian
    from .torch_shim import hea_template
    rng = np.random.default_rng(seed)
    items = []
    for _ in range(ncirc):
        n = int(rng.integers(qmin, qmax + 1))
        layers = int(rng.integers(lmin, lmax + 1))
        pc = hea_template(n, layers)
        params = rng.uniform(-math.pi, math.pi, pc.nparams)
        terms = zz_x_hamiltonian(n, rng.standard_normal(n - 1), rng.standard_normal(n))
        items.append((pc, params, terms))
    return items
