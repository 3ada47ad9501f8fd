"""Segments of the host-resident (out-of-core) runner, on the CPU: every
gate runs exactly once, inside a segment whose local set holds all its
qubits; gates that share a qubit keep their order; the reordered list gives
the same state as the circuit (FP64 oracle)."""
import numpy as np
import pytest

import oracle
from subquokka_dev_b200 import Circuit, circuits, make_gate, ooc_segments


def random_mixed(n, ngates, seed):
    rng = np.random.default_rng(seed)
    gs = []
    for _ in range(ngates):
        k = rng.integers(6)
        if k == 0:
            gs.append(make_gate("H", [int(rng.integers(n))]))
        elif k == 1:
            gs.append(make_gate("RX", [int(rng.integers(n))], float(rng.uniform(-3, 3))))
        elif k == 2:
            a, b = sorted(int(x) for x in rng.choice(n, 2, replace=False))
            gs.append(make_gate("CP", [a, b], float(rng.uniform(-3, 3))))
        elif k == 3:
            a, b = sorted(int(x) for x in rng.choice(n, 2, replace=False))
            gs.append(make_gate("RZZ", [a, b], float(rng.uniform(-3, 3))))
        elif k == 4:
            a, b = sorted(int(x) for x in rng.choice(n, 2, replace=False))
            gs.append(make_gate("SWAP", [a, b]))
        else:
            q = [int(x) for x in rng.choice(n, 4, replace=False)]
            gs.append(make_gate("VSWAP", sorted(q[:2]) + sorted(q[2:])))
    return Circuit(gs)


CASES = [("random_u3_cz", 14, 10), ("random_u3_cz", 14, 12), ("qft", 13, 9), ("mixed", 12, 8), ("mixed", 12, 11)]


def build(kind, n):
    if kind == "random_u3_cz":
        return circuits.random_u3_cz(n, 6, 7)
    if kind == "qft":
        return circuits.qft(n)
    return random_mixed(n, 120, 8)


@pytest.mark.parametrize("kind,n,L", CASES)
def test_segments_are_valid_and_preserve_the_state(kind, n, L):
    circ = build(kind, n)
    segs = ooc_segments(circ, n, L)
    gl = circ.gate_list()
    order = [i for _, idx in segs for i in idx]
    assert sorted(order) == list(range(circ.ngates))
    for mask, idx in segs:
        assert bin(mask).count("1") == L and mask < (1 << n)
        for i in idx:
            qs = {gl[i].q[k] for k in range(gl[i].nq)}
            assert all(mask >> q & 1 for q in qs), (i, qs, bin(mask))
    pos = {g: p for p, g in enumerate(order)}
    qsets = [{gl[i].q[k] for k in range(gl[i].nq)} for i in range(circ.ngates)]
    for i in range(circ.ngates):
        for j in range(i + 1, circ.ngates):
            if qsets[i] & qsets[j]:
                assert pos[i] < pos[j], (i, j)
    init = circuits.random_state(n, 11)
    a = oracle.apply_circuit(init, n, circ)
    b = oracle.apply_circuit(init, n, Circuit([gl[i] for i in order]))
    assert np.abs(a - b).max() <= 1e-12


def test_light_cone_keeps_segment_counts_low():
    # a brick circuit's far qubits reach the others only through the CZ
    # light cone, so a few segments cover 20 layers
    assert len(ooc_segments(circuits.random_u3_cz(34, 20, 1), 34, 30)) <= 3
    assert len(ooc_segments(circuits.qft(34), 34, 30)) <= 4


def test_segment_errors():
    from subquokka_dev_b200 import QkError
    with pytest.raises(QkError):
        ooc_segments(Circuit([make_gate("VSWAP", [0, 1, 2, 3])]), 6, 3)   # 4 qubits, 3 local
    with pytest.raises(QkError):
        ooc_segments(Circuit([make_gate("H", [7])]), 6, 4)
