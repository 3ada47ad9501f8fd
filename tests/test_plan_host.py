"""Host side of the fused planner (no GPU): pass counts and option checks."""
import numpy as np
import pytest

import subquokka_dev_b200 as sq
from subquokka_dev_b200 import Plan, circuits, make_gate
from subquokka_dev_b200.engine import Circuit


def test_random30_is_far_fewer_passes_than_gates():
    c = circuits.random_u3_cz(30, 20, 2030)
    passes, ops, remaps = Plan(c, 30, "c128").stats()
    assert c.ngates == 890
    # U3 pairs fold into the CZ after them: fewer program ops than gates
    assert passes <= 45 and ops <= c.ngates // 2 and remaps < ops


def test_diagonal_gates_join_any_pass():
    # CP gates on qubits outside any tile are diagonal: one pass holds them all
    n = 20
    c = Circuit([make_gate("CP", [a, a + 1], 0.1 * a) for a in range(n - 1)] +
                [make_gate("RZ", [q], 0.3) for q in range(n)] + [make_gate("RZZ", [3, 19], 0.2)])
    assert Plan(c, n, "c128").stats()[0] == 1


def test_program_op_reductions():
    # consecutive one-qubit ops multiply into one, two pending dense ops fold
    # into the two-qubit op after them, one pending dense op folds into a
    # diagonal op or CX as a conditioned 2x2: the 26-qubit HEA forward pass
    # (924 gates) and the 30-qubit brick circuit (890 gates) need far fewer
    # program ops than gates
    from subquokka_dev_b200.torch_shim import hea_template
    pc = hea_template(26, 12)
    c, _ = pc.bind(np.random.default_rng(26).uniform(-np.pi, np.pi, pc.nparams))
    assert c.ngates == 924
    passes, ops, _ = Plan(c, 26, "c128").stats()
    assert ops <= 400 and passes <= 30
    brick = circuits.random_u3_cz(30, 20, 2030)
    assert Plan(brick, 30, "c64").stats()[1] <= 420


def test_vswap_is_a_relabelling():
    # H 0, VSWAP, H 1 = H on stored bits 0 and 15 in one pass, then one
    # permutation pass that brings the state into the circuit's layout
    c = Circuit([make_gate("H", [0]), make_gate("VSWAP", [0, 1, 14, 15]), make_gate("H", [1])])
    p, ops, _ = Plan(c, 16, "c128").stats()
    assert p == 2


def test_group_plan_ignores_group_bounds():
    c = Circuit([make_gate("H", [q]) for q in range(6)] + [make_gate("VSWAP", [0, 1, 8, 9])] +
                [make_gate("U1", [q], coeff=[[0, 1], [1, 0]]) for q in range(4)], [6, 1, 4])
    assert Plan(c, 12, "c128", groups=True).stats()[0] == 2


def test_many_vswaps_cost_at_most_two_rounds():
    # 40 VSWAP_2_2 among compute groups: the restoring permutation is two
    # rounds of disjoint bit swaps whatever the number of VSWAPs
    n = 20
    sub = sq.chunk_groups(circuits.qft(n), n, 6)
    nv = sum(1 for i in range(sub.ngates) if sub.gates[i].kind == sq.engine.GATE_KINDS["VSWAP"])
    assert nv >= 20
    plain = Plan(circuits.qft(n), n, "c128").stats()[0]
    assert Plan(sub, n, "c128", groups=True).stats()[0] <= plain + 2 * 3


@pytest.mark.parametrize("dtype,tile,reg", [("c128", 13, 3), ("c128", 13, 4), ("c128", 12, 5), ("c64", 12, 5), ("c128", 12, 0)])
def test_bad_options_rejected(dtype, tile, reg):
    c = circuits.qft(14)
    if reg == 0:
        Plan(c, 14, dtype, tile, reg)  # defaults fill zero fields
        return
    with pytest.raises(sq.QkError):
        Plan(c, 14, dtype, tile, reg)


def test_plan_rejects_bad_qubits():
    c = Circuit([make_gate("H", [20])])
    with pytest.raises(sq.QkError):
        Plan(c, 10, "c128")


def apply_block(state, n, qubits, u):
    """numpy: apply a 64 x 64 unitary on the given six qubits (local bit b = qubits[b])."""
    psi = state.reshape([2] * n)  # axis n-1-q is qubit q
    axes = [n - 1 - q for q in reversed(qubits)]  # block index bit b = qubit qubits[b]: most significant first
    t = np.moveaxis(psi, axes, list(range(6))).reshape(64, -1)
    t = u @ t
    return np.moveaxis(t.reshape([2] * 6 + [2] * (n - 6)), list(range(6)), axes).reshape(-1)


def idle_qubits(u):
    """Local bits b on which the 64 x 64 unitary u acts as the identity."""
    idle = []
    for b in range(6):
        t = u.reshape([2] * 12)          # axes 0-5: row bits 5..0, axes 6-11: column bits 5..0
        a_row, a_col = 5 - b, 11 - b
        blocks = [[t.take(i, a_row).take(j, a_col - 1) for j in range(2)] for i in range(2)]
        if np.allclose(blocks[0][1], 0, atol=1e-12) and np.allclose(blocks[1][0], 0, atol=1e-12) \
                and np.allclose(blocks[0][0], blocks[1][1], atol=1e-12):
            idle.append(b)
    return idle


@pytest.mark.parametrize("width", [5, 6])
@pytest.mark.parametrize("seed", [1, 2])
def test_dense_fuser_blocks_reproduce_the_circuit(seed, width):
    import oracle
    from test_gpu_fused import random_circuit
    n = 12
    circ = random_circuit(n, 150, seed)
    p = Plan(circ, n, "c64", fuse_width=width)
    nb = p.stats()[0]
    s = circuits.random_state(n, seed)
    out = s.copy()
    for k in range(nb):
        qs, u, perm = p.dense_block(k)
        if perm:
            out = oracle.apply_circuit(out, n, Circuit([make_gate("VSWAP", qs)]))
        else:
            assert np.allclose(u.conj().T @ u, np.eye(64), atol=1e-12)
            assert len(idle_qubits(u)) >= 6 - width     # width 5: one padded, idle qubit
            out = apply_block(out, n, qs, u)
    assert np.abs(out - oracle.apply_circuit(s, n, circ)).max() < 1e-12


def test_dense_blocks_of_a_subcircuit_file_reproduce_the_circuit():
    # a chunk-grouped file's VSWAPs become renamings inside the dense-block
    # fuser; replaying its blocks (permutation blocks as VSWAPs) on the CPU
    # gives the flat circuit's state
    import oracle
    n = 13
    circ = circuits.random_u3_cz(n, 6, 4)
    sub = sq.chunk_groups(circ, n, 5)
    p = Plan(sub, n, "c64", groups=True, fuse_width=6)
    s = circuits.random_state(n, 6)
    out = s.copy()
    nperm = 0
    for k in range(p.stats()[0]):
        qs, u, perm = p.dense_block(k)
        if perm:
            nperm += 1
            out = oracle.apply_circuit(out, n, Circuit([make_gate("VSWAP", qs)]))
        else:
            out = apply_block(out, n, qs, u)
    assert nperm <= 2 * 6          # the final restore only, at most two rounds
    assert np.abs(out - oracle.apply_circuit(s, n, circ)).max() < 1e-12


def test_fuse_width_must_be_5_or_6():
    c = circuits.random_u3_cz(14, 2, 3)
    for w in (1, 4, 7):
        with pytest.raises(sq.QkError):
            Plan(c, 14, "c64", fuse_width=w)
    assert Plan(c, 14, "c64", fuse_width=5).stats()[0] > Plan(c, 14, "c64", fuse_width=6).stats()[0]


def test_dense_fuser_block_count():
    c = circuits.random_u3_cz(33, 24, 33)
    nb = Plan(c, 33, "c64", fuse_width=6).stats()[0]
    assert nb < c.ngates / 4
    # complex128 blocks (int8 tensor cores) use the same fuser
    assert Plan(c, 33, "c128", fuse_width=6).stats()[0] == nb
    with pytest.raises(sq.QkError):
        Plan(circuits.random_u3_cz(11, 2, 3), 11, "c128", fuse_width=6)
