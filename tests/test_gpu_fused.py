"""Parity of the fused-pass path (qk_plan_*) with the oracle and with the
per-gate path.  complex128 <= 1e-12; complex64 within FP32 rounding."""
import numpy as np
import pytest

import oracle
from subquokka_dev_b200 import Circuit, Plan, StateVector, circuits, make_gate

pytestmark = pytest.mark.gpu

KINDS1 = ["H", "X", "Y", "Z", "P", "RX", "RY", "RZ", "U1"]
KINDS2 = ["U2", "SWAP", "CP", "RZZ"]


def zero(n):
    s = np.zeros(1 << n, np.complex128)
    s[0] = 1
    return s


def run_plan(n, circ, init, dtype="c128", tile=0, reg=0, groups=False, fuse_width=0):
    plan = Plan(circ, n, dtype, tile, reg, groups, fuse_width)
    with StateVector(n, dtype) as sv:
        if init is not None:
            sv.upload(init)
        plan.apply(sv)
        out = sv.download()
    plan.close()
    return out


def random_circuit(n, ngates, seed, vswap=True):
    rng = np.random.default_rng(seed)
    gates = []
    for _ in range(ngates):
        r = rng.random()
        if vswap and r < 0.03:
            qs = [int(x) for x in rng.choice(n, 4, replace=False)]
            gates.append(make_gate("VSWAP", qs))
        elif r < 0.55:
            k = KINDS1[rng.integers(len(KINDS1))]
            q = [int(rng.integers(n))]
            if k == "U1":
                z = rng.standard_normal((2, 2)) + 1j * rng.standard_normal((2, 2))
                gates.append(make_gate(k, q, coeff=np.linalg.qr(z)[0]))
            else:
                gates.append(make_gate(k, q, rng.uniform(-4, 4)))
        else:
            k = KINDS2[rng.integers(len(KINDS2))]
            q = sorted(int(x) for x in rng.choice(n, 2, replace=False))
            if k == "U2":
                z = rng.standard_normal((4, 4)) + 1j * rng.standard_normal((4, 4))
                gates.append(make_gate(k, q, coeff=np.linalg.qr(z)[0]))
            else:
                gates.append(make_gate(k, q, rng.uniform(-4, 4)))
    return Circuit(gates)


@pytest.mark.parametrize("tile,reg", [(0, 0), (6, 2), (7, 2), (8, 3), (10, 3), (12, 3), (11, 2), (4, 2)])
def test_random_gate_mix_c128(tile, reg):
    n = 15
    circ = random_circuit(n, 300, 11 + tile + reg)
    init = circuits.random_state(n, 3)
    ref = oracle.apply_circuit(init, n, circ)
    assert np.abs(run_plan(n, circ, init, "c128", tile, reg) - ref).max() <= 1e-12


@pytest.mark.parametrize("tile,reg", [(0, 0), (13, 4), (9, 4), (6, 2), (12, 3)])
def test_random_gate_mix_c64(tile, reg):
    n = 15
    circ = random_circuit(n, 300, 21 + tile + reg)
    init = circuits.random_state(n, 4)
    ref = oracle.apply_circuit(init, n, circ)
    assert np.abs(run_plan(n, circ, init, "c64", tile, reg) - ref).max() <= 2e-6


@pytest.mark.parametrize("n", [3, 5, 9, 12, 13])
def test_small_states(n):
    circ = random_circuit(n, 120, 100 + n, vswap=n >= 4)
    init = circuits.random_state(n, 5)
    ref = oracle.apply_circuit(init, n, circ)
    assert np.abs(run_plan(n, circ, init) - ref).max() <= 1e-12
    assert np.abs(run_plan(n, circ, init, "c64") - ref).max() <= 2e-6


def test_benchmark_circuit_families():
    n = 18
    for circ in (circuits.random_u3_cz(n, 10, 7), circuits.qft(n), circuits.hea(n, 4, 8)[0]):
        ref = oracle.apply_circuit(zero(n), n, circ)
        assert np.abs(run_plan(n, circ, None) - ref).max() <= 1e-12


def test_group_plan_matches_flat():
    n = 14
    circ = random_circuit(n, 200, 77)
    sizes = []
    left = circ.ngates
    rng = np.random.default_rng(1)
    while left:
        k = int(min(left, rng.integers(1, 20)))
        sizes.append(k)
        left -= k
    grouped = Circuit(circ.gate_list(), sizes)
    init = circuits.random_state(n, 6)
    ref = oracle.apply_circuit(init, n, circ)
    assert np.abs(run_plan(n, grouped, init, groups=True) - ref).max() <= 1e-12


def test_plan_reuse_and_large_state():
    # one plan applied twice on a 30-qubit state equals the per-gate path
    n = 28
    circ = circuits.random_u3_cz(n, 6, 9)
    plan = Plan(circ, n, "c128")
    with StateVector(n) as a, StateVector(n) as b:
        plan.apply(a)
        plan.apply(a)
        b.apply(circ)
        b.apply(circ)
        x, y = a.download(), b.download()
    assert np.abs(x - y).max() <= 1e-12


def fidelity_err(out, ref):
    ov = np.vdot(ref, out)
    return 1 - abs(ov) ** 2 / (np.vdot(ref, ref).real * np.vdot(out, out).real)


@pytest.mark.parametrize("n,width", [(12, 6), (14, 6), (17, 6), (13, 5), (17, 5)])
def test_tensor_core_dense_blocks(n, width):
    # 6-qubit blocks (or 5-qubit blocks padded to 6) as 64 x 64 complex
    # contractions on tcgen05 (3 x BF16, FP32 accumulate): 1 - F <= 1e-6
    # against the FP64 oracle
    circ = random_circuit(n, 200, 300 + n)
    init = circuits.random_state(n, 31)
    ref = oracle.apply_circuit(init, n, circ)
    out = run_plan(n, circ, init, "c64", fuse_width=width)
    assert fidelity_err(out, ref) <= 1e-6
    assert np.abs(out - ref).max() <= 5e-5


def test_tensor_core_random_circuit_family():
    n = 20
    circ = circuits.random_u3_cz(n, 8, 40)
    ref = oracle.apply_circuit(zero(n), n, circ)
    out = run_plan(n, circ, None, "c64", fuse_width=6)
    assert fidelity_err(out, ref) <= 1e-6


def block_circuit(blocks, seed):
    """Gates that the fuser groups into exactly the given 6-qubit blocks."""
    rng = np.random.default_rng(seed)
    gates = []
    for qs in blocks:
        qs = sorted(qs)
        for a, b in zip(qs, qs[1:]):
            gates.append(make_gate("CP", [a, b], float(rng.uniform(0, 6))))
        for q in qs:
            gates.append(make_gate("U1", [q], coeff=circuits.u3_matrix(*rng.uniform(0, 2 * np.pi, 3))))
        for a, b in zip(qs, qs[1:]):
            gates.append(make_gate("CP", [a, b], float(rng.uniform(0, 6))))
    return Circuit(gates)


@pytest.mark.parametrize("n,blocks", [
    (16, [[0, 1, 2, 3, 4, 5], [6, 7, 8, 9, 10, 11]]),          # first block owns qubit 0
    (16, [[6, 7, 8, 9, 10, 11], [0, 1, 2, 3, 4, 5]]),          # second block owns qubit 0
    (16, [[0, 1, 2, 8, 9, 10], [0, 3, 4, 5, 12, 13]]),         # both, overlapping
    (16, [[3, 4, 5, 6, 7, 8], [9, 10, 11, 12, 13, 14]]),       # neither
    (16, [[2, 5, 7, 9, 11, 13], [1, 4, 6, 8, 10, 15]]),        # interleaved qubits
    (13, [[1, 2, 3, 4, 5, 6], [7, 8, 9, 10, 11, 12]]),         # one supertile
    (15, [[0, 1, 2, 3, 4, 5], [6, 7, 8, 9, 10, 11], [3, 4, 5, 12, 13, 14]]),  # a pair and a single
])
def test_tensor_core_block_sequences(n, blocks):
    # blocks on chosen qubit sets: both operand layouts (qubit 0 in the first,
    # the second, both or neither block), interleaved qubits, a 13-qubit
    # state (one supertile) and a trailing block
    circ = block_circuit(blocks, 7 + n)
    p = Plan(circ, n, "c64", fuse_width=6)
    got = [p.dense_block(k)[0] for k in range(p.stats()[0])]
    assert len(got) == len(blocks) and got[:2] == blocks[:2]
    p.close()
    init = circuits.random_state(n, 8)
    ref = oracle.apply_circuit(init, n, circ)
    out = run_plan(n, circ, init, "c64", fuse_width=6)
    assert fidelity_err(out, ref) <= 1e-6
    assert np.abs(out - ref).max() <= 5e-5


# complex128 dense blocks: the same blocks as exact integer contractions on the
# int8 tensor cores (seven 8-bit digits an operand row, 28 digit products,
# int32 accumulate, FP64 recombination): within 1e-12 of the FP64 oracle
TOL_C128_TC = 1e-12


@pytest.mark.parametrize("n,width", [(12, 6), (13, 6), (14, 6), (17, 6), (13, 5), (18, 5)])
def test_tensor_core_c128_dense_blocks(n, width):
    circ = random_circuit(n, 200, 500 + n)
    init = circuits.random_state(n, 41)
    ref = oracle.apply_circuit(init, n, circ)
    out = run_plan(n, circ, init, "c128", fuse_width=width)
    assert np.abs(out - ref).max() <= TOL_C128_TC
    assert fidelity_err(out, ref) <= 1e-15   # the FP64 rounding floor of fidelity_err


def test_tensor_core_c128_random_circuit_family():
    # from |0>: early blocks see rows of zeros
    n = 20
    circ = circuits.random_u3_cz(n, 8, 40)
    ref = oracle.apply_circuit(zero(n), n, circ)
    out = run_plan(n, circ, None, "c128", fuse_width=6)
    assert np.abs(out - ref).max() <= TOL_C128_TC


@pytest.mark.parametrize("n,blocks", [
    (16, [[0, 1, 2, 3, 4, 5], [6, 7, 8, 9, 10, 11]]),
    (16, [[6, 7, 8, 9, 10, 11], [0, 1, 2, 3, 4, 5]]),
    (16, [[0, 1, 2, 8, 9, 10], [0, 3, 4, 5, 12, 13]]),
    (16, [[3, 4, 5, 6, 7, 8], [9, 10, 11, 12, 13, 14]]),
    (16, [[2, 5, 7, 9, 11, 13], [1, 4, 6, 8, 10, 15]]),
    (12, [[0, 1, 2, 3, 4, 5], [6, 7, 8, 9, 10, 11]]),          # one supertile
    (15, [[0, 1, 2, 3, 4, 5], [6, 7, 8, 9, 10, 11], [3, 4, 5, 12, 13, 14]]),
])
def test_tensor_core_c128_block_sequences(n, blocks):
    circ = block_circuit(blocks, 9 + n)
    p = Plan(circ, n, "c128", fuse_width=6)
    got = [p.dense_block(k)[0] for k in range(p.stats()[0])]
    assert len(got) == len(blocks) and got[:2] == blocks[:2]
    p.close()
    init = circuits.random_state(n, 10)
    ref = oracle.apply_circuit(init, n, circ)
    out = run_plan(n, circ, init, "c128", fuse_width=6)
    assert np.abs(out - ref).max() <= TOL_C128_TC


def test_tensor_core_c128_wide_dynamic_range():
    # amplitudes spread over 2^-200 .. 1 and exact zeros: each row of a
    # supertile is scaled by its own largest entry, so small rows keep their
    # relative precision
    n = 14
    rng = np.random.default_rng(12)
    init = circuits.random_state(n, 13) * np.exp2(-rng.integers(0, 200, 1 << n))
    init[rng.random(1 << n) < 0.1] = 0
    circ = block_circuit([[1, 3, 5, 7, 9, 11], [0, 2, 4, 6, 8, 10]], 14)
    ref = oracle.apply_circuit(init, n, circ)
    out = run_plan(n, circ, init, "c128", fuse_width=6)
    assert np.abs(out - ref).max() <= 1e-15
    # the whole state scaled by 2^-900: the same relative error
    tiny = circuits.random_state(n, 15) * np.exp2(-900)
    ref = oracle.apply_circuit(tiny, n, circ)
    out = run_plan(n, circ, tiny, "c128", fuse_width=6)
    assert np.abs(out - ref).max() <= 1e-12 * np.abs(ref).max()


def test_tensor_core_c128_repeated_large_state():
    # a 28-qubit state (4 GiB, 16k supertiles a block spread over every SM),
    # the circuit applied three times over: every run must match the fused
    # complex128 passes; a race between the kernel's pipeline stages shows
    # up here as an error far above 1e-12
    import torch
    n = 28
    circ = circuits.random_u3_cz(n, 6, 2828)
    tc = Plan(circ, n, "c128", fuse_width=6)
    ps = Plan(circ, n, "c128")
    with StateVector(n, "c128") as a, StateVector(n, "c128") as b:
        for rep in range(3):
            tc.apply(a)
            ps.apply(b)
            a.synchronize()
            b.synchronize()
            d = float((a.as_torch() - b.as_torch()).abs().max())
            assert d <= TOL_C128_TC, (rep, d)
    tc.close()
    ps.close()
    torch.cuda.empty_cache()


@pytest.mark.parametrize("form", ["per_gate", "passes_c128", "tensor_core_c128", "tensor_core_c64"])
def test_known_answers_every_form(form):
    # the analytic answers the reference's own circuits have, through every
    # form: H^n |0> = 0.70710678118^n everywhere (the reference's literal),
    # RX(pi)^n |0> = (-i)^n |1...1>, QFT |0> uniform
    n = 14
    cases = [
        (Circuit([make_gate("H", [q]) for q in range(n)]), lambda s: np.full_like(s, 0.70710678118 ** n)),
        (Circuit([make_gate("RX", [q], np.pi) for q in range(n)]),
         lambda s: np.where(np.arange(s.size) == s.size - 1, (-1j) ** n, 0)),
        (circuits.qft(n), lambda s: np.full_like(s, 0.70710678118 ** n)),
    ]
    dtype = "c64" if form.endswith("c64") else "c128"
    tol = 1e-6 if dtype == "c64" else 1e-12
    for circ, want in cases:
        with StateVector(n, dtype) as sv:
            if form == "per_gate":
                sv.apply(circ)
            else:
                plan = Plan(circ, n, dtype, fuse_width=6 if form.startswith("tensor") else 0)
                plan.apply(sv)
                plan.close()
            out = sv.download()
        assert np.abs(out - want(out)).max() <= tol, form
