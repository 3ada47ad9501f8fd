"""Chunk grouping (the subcircuitFinder role): the subcircuit files that
qk_circuit_chunk_groups writes keep the finder's contract and compute the
flat circuit's state, in the oracle and in the reference's own subcircuit
runner (src/MEM_Runner.cpp:136-185) where its build is present."""
import os
import subprocess

import numpy as np
import pytest

import oracle
import subquokka_dev_b200 as sq
from subquokka_dev_b200 import Circuit, chunk_groups, circuits, make_gate
from test_gpu_fused import random_circuit

VSWAP = sq.engine.GATE_KINDS["VSWAP"]


def check_contract(sub: Circuit, c: int):
    """Compute groups on positions < c with ascending targets; VSWAP groups
    of one VSWAP_1_1 / VSWAP_2_2 with a < b < c <= x < y."""
    k = 0
    for gi in range(sub.ngroups):
        size = sub.group_sizes[gi]
        assert size > 0
        for j in range(size):
            g = sub.gates[k + j]
            qs = [g.q[i] for i in range(g.nq)]
            if g.kind == VSWAP:
                h = g.nq // 2
                assert size == 1 and h in (1, 2)
                lo, hi = qs[:h], qs[h:]
                assert lo == sorted(lo) and hi == sorted(hi) and max(lo) < c <= min(hi)
            else:
                assert max(qs) < c and qs == sorted(set(qs)), (qs, c)
        k += size


CASES = [("qft", lambda n: circuits.qft(n)),
         ("u3cz", lambda n: circuits.random_u3_cz(n, 5, n)),
         ("mixed", lambda n: random_circuit(n, 160, 40 + n))]


@pytest.mark.parametrize("name,make", CASES)
@pytest.mark.parametrize("n,c", [(10, 2), (10, 4), (11, 5), (12, 12)])
def test_chunk_groups_keep_contract_and_state(name, make, n, c):
    circ = make(n)
    sub = chunk_groups(circ, n, c)
    check_contract(sub, c)
    init = circuits.random_state(n, 5)
    ref = oracle.apply_circuit(init, n, circ)
    assert np.abs(oracle.apply_circuit(init, n, sub) - ref).max() <= 1e-12
    # the text round-trips through the parser
    again = Circuit.parse(sub.to_text(True), 1, n)
    assert again.ngates == sub.ngates and list(again.group_sizes) == list(sub.group_sizes)


@pytest.mark.skipif(not oracle.have_reference(), reason="reference build (oracle/_ref) absent")
@pytest.mark.parametrize("name,make", CASES)
def test_reference_subcircuit_runner_accepts_chunk_groups(name, make):
    n, c = 12, 5
    circ = make(n)
    sub = chunk_groups(circ, n, c)
    init = circuits.random_state(n, 8)
    # the flat file's arbitrary VSWAPs are outside the reference's own
    # VSWAP forms, so the flat state comes from the pinned oracle
    flat = oracle.apply_circuit(init, n, circ)
    grouped, _ = oracle.run_reference(n, sub.to_text(True), 1, init, chunk_qbit=c)
    assert np.abs(grouped - flat).max() <= 1e-12


def test_u2_written_in_swapped_basis():
    # a U2 whose qubits land in descending positions is rewritten with its
    # matrix in the swapped basis (the reference asserts targ0 < targ1)
    n, c = 6, 2
    z = np.random.default_rng(3).standard_normal((4, 4, 2)) @ [1, 1j]
    u = np.linalg.qr(z)[0]
    circ = Circuit([make_gate("SWAP", [0, 5]), make_gate("U2", [0, 1], coeff=u), make_gate("H", [3])])
    sub = chunk_groups(circ, n, c)
    check_contract(sub, c)
    init = circuits.random_state(n, 2)
    assert np.abs(oracle.apply_circuit(init, n, sub) - oracle.apply_circuit(init, n, circ)).max() <= 1e-12


def test_input_vswaps_are_absorbed():
    n = 9
    circ = Circuit([make_gate("H", [0]), make_gate("VSWAP", [0, 1, 7, 8]), make_gate("CP", [0, 1], 0.3),
                    make_gate("VSWAP", [2, 6]), make_gate("RX", [2], 0.7)])
    sub = chunk_groups(circ, n, 4)
    check_contract(sub, 4)
    init = circuits.random_state(n, 4)
    assert np.abs(oracle.apply_circuit(init, n, sub) - oracle.apply_circuit(init, n, circ)).max() <= 1e-12


def test_qft30_vswap_count():
    # 30-qubit QFT, 12-qubit chunks: fewer VSWAPs before the final restore
    # than the reference finder's 42 for the same circuit
    sub = chunk_groups(circuits.qft(30), 30, 12)
    check_contract(sub, 12)
    kinds = [(sub.gates[i].kind, sub.gates[i].nq) for i in range(sub.ngates)]
    last_compute = max(i for i, (k, _) in enumerate(kinds) if k not in (VSWAP, sq.engine.GATE_KINDS["SWAP"]))
    assert sum(1 for k, _ in kinds[:last_compute] if k == VSWAP) < 42


def test_empty_and_small_circuits():
    empty = chunk_groups(Circuit([]), 5, 2)
    assert empty.ngates == 0 and empty.to_text(True) == ""
    assert Circuit.parse(empty.to_text(True), 1, 5).ngates == 0
    one = chunk_groups(Circuit([make_gate("H", [0]), make_gate("RX", [0], 0.3)]), 1, 1)
    assert one.ngates == 2 and one.ngroups == 1
    # chunk = whole state: no VSWAP, the final SWAPs as in-chunk SWAP gates
    full = chunk_groups(circuits.qft(6), 6, 6)
    check_contract(full, 6)
    init = circuits.random_state(6, 3)
    assert np.abs(oracle.apply_circuit(init, 6, full) - oracle.apply_circuit(init, 6, circuits.qft(6))).max() <= 1e-12


def test_chunk_groups_errors():
    circ = Circuit([make_gate("CP", [0, 1], 0.1)])
    for n, c in ((0, 1), (4, 0), (4, 5)):
        with pytest.raises(sq.QkError):
            chunk_groups(circ, n, c)
    with pytest.raises(sq.QkError):
        chunk_groups(circ, 4, 1)          # a two-qubit gate needs two chunk positions
    with pytest.raises(sq.QkError):
        chunk_groups(Circuit([make_gate("H", [5])]), 4, 2)


def test_finder_cli(tmp_path):
    # quokka_finder circuit.txt [mode] [sub.txt] --chunk K, the reference
    # finder's argument order (subcircuitFinder/finder.cpp:771-784)
    exe = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                       "subquokka_dev_b200", "bin", "quokka_finder")
    n = 11
    circ = circuits.qft(n)
    (tmp_path / "c.txt").write_text(circ.to_text(False))
    r = subprocess.run([exe, str(tmp_path / "c.txt"), "1", str(tmp_path / "s.txt"), "--chunk", "4"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert "11 qubits, chunk 4" in r.stdout
    sub = Circuit.parse((tmp_path / "s.txt").read_text(), 1, n)
    check_contract(sub, 4)
    init = circuits.random_state(n, 1)
    assert np.abs(oracle.apply_circuit(init, n, sub) - oracle.apply_circuit(init, n, circ)).max() <= 1e-12
    bad = subprocess.run([exe, str(tmp_path / "missing.txt")], capture_output=True, text=True)
    assert bad.returncode == 1 and "cannot open" in bad.stderr
