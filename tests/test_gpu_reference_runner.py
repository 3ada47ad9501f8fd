"""The drop-in, end to end: the reference's own CLI and Simulator
(src/main.cpp, src/simulator.cpp) with this engine in its runner_type=GPU slot
(oracle/_ref/Quokka_gpu: the reference's objects, a copy of simulator.cpp
with the GPU stub replaced by GPU_Runner, subquokka_dev_b200/runner, and
libquokka_gpu.so).  `Quokka_gpu -i gpu.ini -c circuit.txt` parses the
reference's golden circuits with the reference's MEM parser, runs them on the
GPU through GPU_Runner::run, and its dump must match the reference's own
final state (tests/golden, made by the unmodified reference) to 1e-12.
"""
import os
import re
import subprocess

import numpy as np
import pytest

import golden_util as gu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "oracle", "_ref", "Quokka_gpu")

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.path.exists(EXE), reason="oracle/_ref/Quokka_gpu not built")]

CASES = ["g1_H", "g1_X", "g1_Y", "g1_Z", "g1_P", "g1_RX", "g1_RY", "g1_RZ", "g1_U1", "g2_CP", "g2_RZZ",
         "g2_SWAP", "g2_U2", "vswap22", "qft12", "sub12", "rand10", "hea8", "qft21", "sub21"]


def run_quokka_gpu(tmp_path, rec, extra=""):
    n = rec["n"]
    init = gu.initial_state(rec)
    ini_lines = [f"total_qbit={n}", f"file_qbit={int(rec['file_qbit'])}", f"chunk_qbit={int(rec['chunk_qbit'])}",
                 "runner_type=GPU", f"is_subcircuit={rec['is_subcircuit']}"]
    ip = tmp_path / "init.bin"
    np.ascontiguousarray(init, dtype=np.complex128).tofile(ip)
    ini_lines.append(f"init_file={ip}")
    ini_lines += [x for x in extra.split("\n") if x]
    (tmp_path / "gpu.ini").write_text("[system]\n" + "\n".join(ini_lines) + "\n")
    (tmp_path / "circuit.txt").write_text(rec["circuit"])
    r = subprocess.run([EXE, "-i", str(tmp_path / "gpu.ini"), "-c", str(tmp_path / "circuit.txt")],
                       capture_output=True, text=True, timeout=300, cwd=tmp_path)
    return r


@pytest.mark.parametrize("name", CASES)
def test_reference_cli_with_gpu_runner_matches_golden(tmp_path, name):
    rec = gu.load(name)
    out = tmp_path / "state.bin"
    r = run_quokka_gpu(tmp_path, rec, f"dump_file={out}\ndump_format=bin")
    assert r.returncode == 0, r.stdout + r.stderr
    assert "GPU Mode" in r.stdout
    assert re.search(r"^[0-9.eE+-]+s$", r.stdout, re.M), r.stdout   # Simulator::run's "<sec>s"
    final = np.fromfile(out, dtype=np.complex128)
    assert final.size == 1 << rec["n"]
    assert gu.compare(rec, final) <= 1e-12


def test_reference_text_dump_through_gpu_runner(tmp_path):
    """dump_file + MPI_testing=1: the reference's own text dump format and
    file name (dump_file[0:3] + rank + ".txt", %.11f), written by GPU_Runner."""
    rec = gu.load("qft12")
    r = run_quokka_gpu(tmp_path, rec, "dump_file=res_gpu.txt\nMPI_testing=1")
    assert r.returncode == 0, r.stdout + r.stderr
    vals = np.loadtxt(tmp_path / "res0.txt")
    final = vals[0::2] + 1j * vals[1::2]
    assert np.abs(final - rec["final"]).max() <= 1e-11   # 11 printed digits


def test_fused_and_complex64_keys_through_gpu_runner(tmp_path):
    """The engine's own .ini keys, which the reference ignores: fuse_width
    (fused passes, complex128, exact) and precision=c64 with 6-qubit tensor-core
    blocks (1 - F <= 1e-6)."""
    rec = gu.load("qft12")
    out = tmp_path / "state.bin"
    r = run_quokka_gpu(tmp_path, rec, f"dump_file={out}\ndump_format=bin\nfuse_width=3")
    assert r.returncode == 0, r.stdout + r.stderr
    assert np.abs(np.fromfile(out, dtype=np.complex128) - rec["final"]).max() <= 1e-12
    r = run_quokka_gpu(tmp_path, rec, f"dump_file={out}\ndump_format=bin\nprecision=c64\nfuse_width=6")
    assert r.returncode == 0, r.stdout + r.stderr
    f = np.fromfile(out, dtype=np.complex128)
    ref = rec["final"]
    fid = abs(np.vdot(ref, f)) ** 2 / (np.vdot(ref, ref).real * np.vdot(f, f).real)
    assert 1 - fid <= 1e-6
