"""Parity of the CUDA path with the reference (golden states) and the oracle.

Bar: complex128 max |delta amp| <= 1e-12 against the reference's complex128
state; complex64 within 2e-6 (FP32 rounding of the stored state).  Every test
calls the engine through the C ABI (libquokka_gpu.so)."""
import os
import subprocess

import numpy as np
import pytest

import oracle
from subquokka_dev_b200 import Circuit, QkError, StateVector, apply_gates_dev, chunk_groups, circuits, make_gate

import golden_util as gu

pytestmark = pytest.mark.gpu

TOL_C128 = 1e-12
TOL_C64 = 2e-6
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "subquokka_dev_b200", "bin", "quokka")


def run_gpu(n, circ, init, dtype="c128", groups=False):
    with StateVector(n, dtype) as sv:
        if init is not None:
            sv.upload(init)
        if groups:
            sv.apply_groups(circ)
        else:
            sv.apply(circ)
        return sv.download()


@pytest.mark.parametrize("name", gu.names())
def test_per_gate_path_matches_reference(name):
    rec = gu.load(name)
    circ = Circuit.parse(rec["circuit"], rec["is_subcircuit"], rec["n"])
    out = run_gpu(rec["n"], circ, gu.initial_state(rec))
    assert gu.compare(rec, out) <= TOL_C128


@pytest.mark.parametrize("name", gu.names())
def test_group_path_matches_reference(name):
    # flat fixtures run as one group per gate: every op kind goes through the tile pass
    rec = gu.load(name)
    circ = Circuit.parse(rec["circuit"], rec["is_subcircuit"], rec["n"])
    out = run_gpu(rec["n"], circ, gu.initial_state(rec), groups=True)
    assert gu.compare(rec, out) <= TOL_C128


@pytest.mark.parametrize("name", gu.names())
def test_c64_path_matches_reference(name):
    rec = gu.load(name)
    circ = Circuit.parse(rec["circuit"], rec["is_subcircuit"], rec["n"])
    init = gu.initial_state(rec)
    assert gu.compare(rec, run_gpu(rec["n"], circ, init, "c64")) <= TOL_C64
    assert gu.compare(rec, run_gpu(rec["n"], circ, init, "c64", groups=True)) <= TOL_C64


def random_gate(rng, kind, qs):
    if kind in ("P", "RX", "RY", "RZ", "CP", "RZZ"):
        return make_gate(kind, qs, rng.uniform(-7, 7))
    if kind in ("U1", "U2"):
        d = 2 if kind == "U1" else 4
        z = rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d))
        q, _ = np.linalg.qr(z)
        return make_gate(kind, qs, coeff=q)
    return make_gate(kind, qs)


@pytest.mark.parametrize("kind", ["H", "X", "Y", "Z", "P", "RX", "RY", "RZ", "U1"])
def test_one_qubit_gate_on_every_qubit(kind):
    n = 13
    rng = np.random.default_rng(sum(map(ord, kind)))
    init = circuits.random_state(n, 7)
    for q in range(n):
        circ = Circuit([random_gate(rng, kind, [q])])
        ref = oracle.apply_circuit(init, n, circ)
        assert np.abs(run_gpu(n, circ, init) - ref).max() <= TOL_C128, q
        assert np.abs(run_gpu(n, circ, init, groups=True) - ref).max() <= TOL_C128, q


@pytest.mark.parametrize("kind", ["U2", "SWAP", "CP", "RZZ"])
def test_two_qubit_gate_on_many_pairs(kind):
    n = 13
    rng = np.random.default_rng(sum(map(ord, kind)))
    init = circuits.random_state(n, 8)
    pairs = [(0, 1), (0, 4), (0, 12), (3, 4), (4, 5), (4, 9), (5, 6), (5, 12), (11, 12), (1, 7)]
    for a, b in pairs:
        circ = Circuit([random_gate(rng, kind, [a, b])])
        ref = oracle.apply_circuit(init, n, circ)
        assert np.abs(run_gpu(n, circ, init) - ref).max() <= TOL_C128, (a, b)
        assert np.abs(run_gpu(n, circ, init, groups=True) - ref).max() <= TOL_C128, (a, b)


@pytest.mark.parametrize("qs", [
    [0, 1, 2, 7, 8, 9], [2, 5, 9, 10, 11, 13], [0, 3, 6, 9, 12, 1, 4, 7],
    [0, 1, 2, 3, 4, 5, 8, 9, 10, 11, 12, 13],      # VSWAP_6_6: does not fit one tile
    [6, 7, 8, 9, 10, 11, 12, 13, 0, 1, 2, 3],
])
def test_vswap_k_k_intended_semantics(qs):
    # VSWAP_k_k = SWAP(q[i], q[k+i]) for i < k (the reference's MEM versions of
    # k >= 3 index the wrong buffer, so the oracle states the documented intent)
    n = 14
    init = circuits.random_state(n, 9)
    circ = Circuit([make_gate("VSWAP", qs)])
    ref = oracle.apply_circuit(init, n, circ)
    k = len(qs) // 2
    swaps = Circuit([make_gate("SWAP", sorted([qs[i], qs[k + i]])) for i in range(k)])
    assert np.abs(oracle.apply_circuit(init, n, swaps) - ref).max() == 0
    assert np.abs(run_gpu(n, circ, init) - ref).max() == 0
    assert np.abs(run_gpu(n, circ, init, groups=True) - ref).max() == 0


def test_qft20_config_matches_oracle():
    # 20-qubit QFT on a seeded random normalised complex128 state, per-gate path
    n = 20
    init = circuits.random_state(n, 20)
    circ = circuits.qft(n)
    ref = oracle.apply_circuit(init, n, circ)
    assert np.abs(run_gpu(n, circ, init) - ref).max() <= TOL_C128


def test_random_circuit_family_matches_oracle():
    n = 16
    circ = circuits.random_u3_cz(n, 6, 30)
    ref = oracle.apply_circuit(gu.initial_state({"n": n, "sampled": False, "init": np.zeros(0)}), n, circ)
    assert np.abs(run_gpu(n, circ, None) - ref).max() <= TOL_C128
    assert np.abs(run_gpu(n, circ, None, groups=True) - ref).max() <= TOL_C128


@pytest.mark.parametrize("dtype,tol", [("c128", TOL_C128), ("c64", TOL_C64)])
@pytest.mark.parametrize("name", ["qft", "u3cz"])
def test_chunk_grouped_file_through_group_path(name, dtype, tol):
    # a subcircuit file from chunk_groups (12-qubit chunks, VSWAP_2_2 /
    # VSWAP_1_1 groups between the compute groups) through the group path:
    # the VSWAPs become renamings and the result is the flat circuit's state
    n = 22
    circ = circuits.qft(n) if name == "qft" else circuits.random_u3_cz(n, 8, 4)
    sub = chunk_groups(circ, n, 12)
    assert sum(1 for i in range(sub.ngates) if sub.gates[i].kind == 14) >= 4
    init = circuits.random_state(n, 12)
    ref = oracle.apply_circuit(init, n, circ)
    assert np.abs(run_gpu(n, sub, init, dtype, groups=True) - ref).max() <= tol


def test_chunk_grouped_file_on_tensor_cores():
    # the same kind of file through tensor-core dense blocks (complex64,
    # 3 x BF16): 1 - F <= 1e-6 against the flat circuit
    from subquokka_dev_b200 import Plan
    n = 20
    circ = circuits.random_u3_cz(n, 8, 5)
    sub = chunk_groups(circ, n, 12)
    init = circuits.random_state(n, 13)
    ref = oracle.apply_circuit(init, n, circ)
    plan = Plan(sub, n, "c64", groups=True, fuse_width=6)
    with StateVector(n, "c64") as sv:
        sv.upload(init)
        plan.apply(sv)
        out = sv.download()
    plan.close()
    ov = np.vdot(ref, out)
    assert 1 - abs(ov) ** 2 / (np.vdot(out, out).real * np.vdot(ref, ref).real) <= 1e-6


def test_chunk_grouped_file_on_int8_tensor_cores():
    # the same file's VSWAPs and groups as complex128 dense blocks on the int8
    # tensor cores (exact digit products): within 1e-12 of the flat circuit
    from subquokka_dev_b200 import Plan
    n = 20
    circ = circuits.random_u3_cz(n, 8, 6)
    sub = chunk_groups(circ, n, 12)
    init = circuits.random_state(n, 14)
    ref = oracle.apply_circuit(init, n, circ)
    plan = Plan(sub, n, "c128", groups=True, fuse_width=6)
    with StateVector(n, "c128") as sv:
        sv.upload(init)
        plan.apply(sv)
        out = sv.download()
    plan.close()
    assert np.abs(out - ref).max() <= 1e-12


def inverse(circ):
    out = []
    for g in reversed(circ.gate_list()):
        if g.kind == 9:  # U1
            m = np.array([g.coeff[2 * k] + 1j * g.coeff[2 * k + 1] for k in range(4)]).reshape(2, 2)
            out.append(make_gate("U1", [g.q[0]], coeff=m.conj().T))
        elif g.kind == 12:  # CP
            out.append(make_gate("CP", [g.q[0], g.q[1]], -g.param))
        else:
            raise ValueError(g.kind)
    return Circuit(out)


@pytest.mark.parametrize("n,layers", [(28, 3), (31, 1)])
def test_large_state_round_trip(n, layers):
    # size-independent property at full scale: C then C^-1 returns |0...0>;
    # n = 31 puts amplitude indices above 2^31
    circ = circuits.random_u3_cz(n, layers, 31)
    inv = inverse(circ)
    with StateVector(n) as sv:
        sv.apply(circ)
        sv.apply(inv)
        out = sv.download()
    assert abs(out[0] - 1) < 1e-10
    assert np.abs(out[1:]).max() < 1e-10


def test_apply_on_caller_device_memory():
    import torch
    n = 12
    circ = circuits.random_u3_cz(n, 3, 5)
    t = torch.zeros(1 << n, dtype=torch.complex128, device="cuda")
    t[0] = 1
    apply_gates_dev(t.data_ptr(), n, "c128", circ, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert np.abs(t.cpu().numpy() - run_gpu(n, circ, None)).max() == 0


def test_cli_dump_matches_reference_golden(tmp_path):
    rec = gu.load("sub12")
    ini = tmp_path / "x.ini"
    ini.write_text(f"[system]\ntotal_qbit={rec['n']}\nfile_qbit=2\nchunk_qbit=6\nrunner_type=GPU\n"
                   f"is_subcircuit=1\ndump_file={tmp_path}/state.bin\ndump_format=bin\n")
    cir = tmp_path / "c.txt"
    # the fixture starts from a random state; run the same circuit from |0> on both sides
    cir.write_text(rec["circuit"])
    r = subprocess.run([CLI, "-i", str(ini), "-c", str(cir)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.splitlines()
    assert lines[0].startswith("[Config File]: ") and lines[1].startswith("[Circuit File]: ")
    assert lines[2] == "GPU Mode" and lines[-1].endswith("s")
    out = np.fromfile(tmp_path / "state.bin", dtype=np.complex128)
    circ = Circuit.parse(rec["circuit"], 1, rec["n"])
    z = np.zeros(1 << rec["n"], np.complex128)
    z[0] = 1
    assert np.abs(out - oracle.apply_circuit(z, rec["n"], circ)).max() <= TOL_C128


@pytest.mark.parametrize("name", ["sub12", "rand10", "sub21"])
def test_cli_init_file_reproduces_reference_golden(tmp_path, name):
    # the fixture's own seeded initial state as init_file (raw complex128),
    # its circuit through the CLI, the final state against the reference's
    rec = gu.load(name)
    init = gu.initial_state(rec)
    init.astype(np.complex128).tofile(tmp_path / "init.bin")
    ini = tmp_path / "x.ini"
    ini.write_text(f"[system]\ntotal_qbit={rec['n']}\nfile_qbit=0\nchunk_qbit=4\nrunner_type=GPU\n"
                   f"is_subcircuit={rec['is_subcircuit']}\ninit_file={tmp_path}/init.bin\n"
                   f"dump_file={tmp_path}/state.bin\ndump_format=bin\n")
    (tmp_path / "c.txt").write_text(rec["circuit"])
    r = subprocess.run([CLI, "-i", str(ini), "-c", str(tmp_path / "c.txt")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert gu.compare(rec, np.fromfile(tmp_path / "state.bin", dtype=np.complex128)) <= TOL_C128


@pytest.mark.parametrize("dtype,tol", [("c128", 0.0), ("c64", 2e-7)])
def test_state_file_round_trip(tmp_path, dtype, tol):
    n = 23   # two 2^22-amplitude chunks
    init = circuits.random_state(n, 3)
    with StateVector(n, dtype) as a, StateVector(n, dtype) as b:
        a.upload(init)
        a.save(tmp_path / "s.bin")
        b.load(tmp_path / "s.bin")
        assert np.abs(b.download() - a.download()).max() == 0
        assert np.abs(np.fromfile(tmp_path / "s.bin", dtype=np.complex128) - init).max() <= tol
    with StateVector(n - 1, dtype) as c:
        with pytest.raises(QkError):
            c.load(tmp_path / "s.bin")        # wrong size
        with pytest.raises(QkError):
            c.load(tmp_path / "missing.bin")


def test_cli_text_dump_format(tmp_path):
    # the reference's dump: dump_file[0:3] + rank + ".txt", "%.11f" per line
    ini = tmp_path / "x.ini"
    ini.write_text("[system]\ntotal_qbit=3\nfile_qbit=1\nchunk_qbit=1\nrunner_type=GPU\nis_subcircuit=0\n"
                   "dump_file=res.txt\nMPI_testing=1\n")
    cir = tmp_path / "c.txt"
    cir.write_text("H 0\nH 1\nH 2\n")
    r = subprocess.run([CLI, "-i", str(ini), "-c", str(cir)], capture_output=True, text=True, cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    vals = (tmp_path / "res0.txt").read_text().split()
    assert len(vals) == 16 and vals[0] == "%.11f" % (0.70710678118 ** 3) and vals[1] == "0.00000000000"


@pytest.mark.parametrize("precision,fuse_width,tol", [("c128", 1, 1e-12), ("c64", 1, 2e-6), ("c64", 5, 5e-5),
                                                     ("c64", 6, 5e-5)])
def test_cli_fused_forms(tmp_path, precision, fuse_width, tol):
    n = 14
    ini = tmp_path / "x.ini"
    ini.write_text(f"[system]\ntotal_qbit={n}\nfile_qbit=2\nchunk_qbit=10\nrunner_type=GPU\nis_subcircuit=0\n"
                   f"precision={precision}\nfuse_width={fuse_width}\ndump_file={tmp_path}/s.bin\ndump_format=bin\n")
    circ = circuits.random_u3_cz(n, 6, 77)
    cir = tmp_path / "c.txt"
    cir.write_text(circ.to_text())
    r = subprocess.run([CLI, "-i", str(ini), "-c", str(cir)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = np.fromfile(tmp_path / "s.bin", dtype=np.complex128)
    z = np.zeros(1 << n, np.complex128)
    z[0] = 1
    assert np.abs(out - oracle.apply_circuit(z, n, circ)).max() <= tol


def test_out_of_memory_is_an_error_not_a_fault():
    from subquokka_dev_b200 import QkError
    with pytest.raises(QkError) as e:
        StateVector(36)                      # 1 TiB complex128
    assert e.value.code == -7
    with StateVector(10) as sv:              # the context is still usable
        sv.apply(circuits.qft(10))


def test_distinct_handles_on_two_host_threads():
    # calls on distinct state handles are thread-safe: two host threads, each
    # with its own state and CUDA stream, run per-gate and fused circuits at
    # the same time and get the oracle's states
    import threading
    import torch
    from subquokka_dev_b200 import Plan
    n = 16
    circs = [circuits.random_u3_cz(n, 6, 70 + k) for k in range(2)]
    inits = [circuits.random_state(n, 80 + k) for k in range(2)]
    refs = [oracle.apply_circuit(oracle.apply_circuit(inits[k], n, circs[k]), n, circs[k]) for k in range(2)]
    out, errs = [None, None], []

    def work(k):
        try:
            stream = torch.cuda.Stream()
            plan = Plan(circs[k], n)
            with StateVector(n) as sv:
                sv.set_stream(stream.cuda_stream)
                for _ in range(5):
                    sv.upload(inits[k])
                    sv.apply(circs[k])          # per-gate path
                    plan.apply(sv)              # fused passes
                out[k] = sv.download()
            plan.close()
        except Exception as e:  # reported below, after both threads end
            errs.append(e)

    th = [threading.Thread(target=work, args=(k,)) for k in range(2)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert not errs, errs
    for k in range(2):
        assert np.abs(out[k] - refs[k]).max() <= 1e-12


@pytest.mark.parametrize("dtype", ["c128", "c64"])
def test_gate_graph_replays_the_per_gate_path(dtype):
    # the per-gate kernels captured as one CUDA graph give the per-gate path's
    # amplitudes bit for bit, launch after launch (SWAP, VSWAP_1_1 and
    # VSWAP_2_2 permutations included)
    n = 13
    gates = list(circuits.qft(n).gate_list())
    gates += [make_gate("VSWAP", [0, 1, 9, 11]), make_gate("VSWAP", [2, 12]), make_gate("SWAP", [3, 7])]
    gates += list(circuits.random_u3_cz(n, 2, 5).gate_list())
    circ = Circuit(gates)
    init = circuits.random_state(n, 6)
    with StateVector(n, dtype) as a, StateVector(n, dtype) as b:
        a.upload(init)
        b.upload(init)
        with b.capture(circ) as g:
            for _ in range(3):
                a.apply(circ)
                g.launch()
                assert np.array_equal(a.download(), b.download())
    ref = init
    for _ in range(3):
        ref = oracle.apply_circuit(ref, n, circ)
    tol = 1e-12 if dtype == "c128" else 2e-5
    with StateVector(n, dtype) as c:
        c.upload(init)
        with c.capture(circ) as g:
            for _ in range(3):
                g.launch()
        assert np.abs(c.download() - ref).max() <= tol
