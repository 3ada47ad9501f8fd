"""Generate the golden fixtures under tests/golden/ by running the UNMODIFIED
reference MEM runner (oracle/_ref/quokka_ref, built from the reference's own
sources by ``make -C oracle ref``).

    python tests/golden/make_golden.py

Each fixture is an .npz holding the circuit text, the .ini segment sizes, the
initial state (or its seed) and the reference's final state (full for small
states; strided samples plus checksums for the 21-qubit ones).  The cases
follow the reference's own MEM gate checks (src/correctness/gate_check_MEM.py:
1-qubit gates on every qubit at small N with small chunks, 2-qubit gates on
every ascending pair, VSWAP_2_2 on chunk/non-chunk pairs) plus whole circuits
in flat and subcircuit format.
"""
from __future__ import annotations

import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from subquokka_dev_b200 import circuits  # noqa: E402
from subquokka_dev_b200.engine import Circuit, gate_line, make_gate  # noqa: E402

ONE_Q = ["H", "X", "Y", "Z", "P", "RX", "RY", "RZ", "U1"]
TWO_Q = ["U2", "SWAP", "CP", "RZZ"]
SAMPLE_STRIDE = 509  # odd stride: samples hit every residue of the low qubits


def haar(rng, d):
    z = (rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d))) / math.sqrt(2)
    q, r = np.linalg.qr(z)
    return q * (np.diag(r) / abs(np.diag(r)))


def one_gate(rng, kind, qubits):
    if kind in ("P", "RX", "RY", "RZ", "CP", "RZZ"):
        return make_gate(kind, qubits, rng.uniform(-2 * math.pi, 2 * math.pi))
    if kind == "U1":
        return make_gate(kind, qubits, coeff=haar(rng, 2))
    if kind == "U2":
        return make_gate(kind, qubits, coeff=haar(rng, 4))
    return make_gate(kind, qubits)


def random_sub(n, chunk, rounds, per_group, seed):
    """Subcircuit-format circuit valid for the reference's MEM runner:
    compute groups whose gates all act below chunk_qbit
    (src/MEM_Runner.cpp:172-183), separated by VSWAP_2_2 / VSWAP_1_1 groups
    that exchange chunk and non-chunk qubits (src/MEM_Runner.cpp:145-170)."""
    rng = np.random.default_rng(seed)
    gates, sizes = [], []
    kinds = ONE_Q + TWO_Q
    for _ in range(rounds):
        for _ in range(per_group):
            k = kinds[rng.integers(len(kinds))]
            if k in TWO_Q:
                qs = sorted(int(x) for x in rng.choice(chunk, 2, replace=False))
            else:
                qs = [int(rng.integers(chunk))]
            gates.append(one_gate(rng, k, qs))
        sizes.append(per_group)
        if rng.random() < 0.75:
            a, b = sorted(int(x) for x in rng.choice(chunk, 2, replace=False))
            c, d = sorted(int(x) for x in rng.choice(np.arange(chunk, n), 2, replace=False))
            gates.append(make_gate("VSWAP", [a, b, c, d]))
        else:
            a = int(rng.integers(chunk))
            c = int(rng.integers(chunk, n))
            gates.append(make_gate("VSWAP", [a, c]))
        sizes.append(1)
    return Circuit(gates, sizes)


def save(name, n, circ, is_sub, chunk, file_qbit, init=None, init_seed=None, sampled=False):
    text = circ.to_text(bool(is_sub))
    final, _ = oracle.run_reference(n, text, is_sub, init=init, chunk_qbit=chunk, file_qbit=file_qbit)
    rec = dict(n=n, circuit=np.array(text), is_subcircuit=is_sub, chunk_qbit=chunk, file_qbit=file_qbit)
    if sampled:
        rec.update(init_seed=init_seed, init_sum=init.sum() if init is not None else 1.0,
                   sample_stride=SAMPLE_STRIDE, final_samples=final[::SAMPLE_STRIDE],
                   final_norm2=np.vdot(final, final).real, final_sum=final.sum(),
                   final_wsum=(final * np.exp(1j * np.arange(final.size) * 1e-3)).sum())
    else:
        rec.update(init=init if init is not None else np.zeros(0, np.complex128), final=final)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **rec)
    print(f"{name}: n={n} gates={circ.ngates} groups={circ.ngroups}")


def main():
    if not oracle.have_reference():
        sys.exit("oracle/_ref/quokka_ref is missing: run `make -C oracle ref` first")
    rng = np.random.default_rng(2024)
    # 1-qubit gates on every qubit, N=3 style small segments (gate_check_MEM.py:16-24)
    for k in ONE_Q:
        n = 5
        circ = Circuit([one_gate(rng, k, [q]) for q in range(n)])
        save(f"g1_{k}", n, circ, 0, 2, 1, init=circuits.random_state(n, 100 + ONE_Q.index(k)))
    # 2-qubit gates on every ascending pair (gate_check_MEM.py:224-301)
    for k in TWO_Q:
        n = 6
        circ = Circuit([one_gate(rng, k, [a, b]) for a in range(n) for b in range(a + 1, n)])
        save(f"g2_{k}", n, circ, 0, 2, 2, init=circuits.random_state(n, 200 + TWO_Q.index(k)))
    # VSWAP_2_2 on chunk x non-chunk pairs (gate_check_MEM.py:307-348)
    set0 = [[0, 1], [0, 2], [1, 2]]
    set1 = [[3, 4], [3, 5], [3, 6], [4, 5], [4, 6], [5, 6]]
    circ = Circuit([make_gate("VSWAP", s0 + s1) for s0 in set0 for s1 in set1])
    save("vswap22", 7, circ, 0, 3, 2, init=circuits.random_state(7, 300))
    # whole circuits
    save("qft12", 12, circuits.qft(12), 0, 6, 2, init=circuits.random_state(12, 400))
    save("sub12", 12, random_sub(12, 6, 12, 8, 401), 1, 6, 2, init=circuits.random_state(12, 402))
    save("rand10", 10, circuits.random_u3_cz(10, 4, 403), 0, 4, 2)
    save("hea8", 8, circuits.hea(8, 3, 404)[0], 0, 3, 1)
    # 21 qubits (the reference's smallest benchmark size): samples + checksums
    init = circuits.random_state(21, 20)
    save("qft21", 21, circuits.qft(21), 0, 12, 3, init=init, init_seed=20, sampled=True)
    init = circuits.random_state(21, 21)
    save("sub21", 21, random_sub(21, 12, 16, 24, 405), 1, 12, 3, init=init, init_seed=21, sampled=True)


if __name__ == "__main__":
    main()
