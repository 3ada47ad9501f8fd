"""Host side of the C ABI (no GPU needed): exports, .ini reader, circuit.txt
parser, coefficient construction, CLI argument handling."""
import os
import re
import subprocess

import numpy as np
import pytest

import subquokka_dev_b200 as sq
from subquokka_dev_b200 import _lib, circuits
from subquokka_dev_b200.engine import Circuit, Config, gate_matrix, make_gate, parse_line

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "quokka_gpu.h")
CLI = os.path.join(ROOT, "subquokka_dev_b200", "bin", "quokka")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(qk_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) <= set(_lib.PROTOTYPES), set(names) - set(_lib.PROTOTYPES)
    assert lib.qk_abi_version() == 3


def test_struct_layouts_match_header():
    import ctypes
    assert ctypes.sizeof(_lib.QkGate) == 4 + 4 + 4 * 12 + 8 + 8 * 32
    assert ctypes.sizeof(_lib.QkConfig) == 10 * 4 + 32 + 256 + 256 + 4


def write(tmp_path, name, text):
    p = tmp_path / name
    p.write_text(text)
    return str(p)


def test_ini_defaults_and_keys(tmp_path):
    # setSEG/setENV defaults (src/simulator.cpp:88-186)
    ini = write(tmp_path, "a.ini", "[system]\ntotal_qbit=20\nchunk_qbit=12\nfile_qbit = 3\nrunner_type=GPU\n")
    c = Config(ini)
    assert (c.total_qbit, c.mpi_qbit, c.file_qbit, c.chunk_qbit) == (20, 0, 3, 12)
    assert c.is_subcircuit == 1 and c.MPI_buffe_size == 16 and c.MPI_testing == 0
    assert c.runner_type == "GPU" and c.dump_file == "" and c.precision == 0 and c.init_file == ""


def test_ini_init_file_key(tmp_path):
    ini = write(tmp_path, "i.ini", "[system]\ntotal_qbit=8\nchunk_qbit=4\ninit_file=/data/start.bin\n")
    assert Config(ini).init_file == "/data/start.bin"


def test_ini_comments_case_and_engine_keys(tmp_path):
    ini = write(tmp_path, "b.ini", "; comment\n# another\n[SYSTEM]\nTotal_Qbit : 0x10 ; inline\n"
                                    "chunk_qbit=4\nis_subcircuit=0\nprecision=c64\nruntime=1\n"
                                    "dump_file=res.txt\ndump_format=bin\nmax_depth=1000\n")
    c = Config(ini)
    assert c.total_qbit == 16 and c.chunk_qbit == 4 and c.is_subcircuit == 0
    assert c.precision == 1 and c.dump_binary == 1 and c.dump_file == "res.txt"


@pytest.mark.parametrize("body,code", [
    ("[system]\ntotal_qbit=4\nchunk_qbit=0\n", -1),        # assert(seg.chunk >= 1)
    ("[system]\ntotal_qbit=4\nfile_qbit=3\nchunk_qbit=2\n", -1),  # assert(N >= file + chunk)
])
def test_ini_reference_asserts_become_errors(tmp_path, body, code):
    with pytest.raises(sq.QkError) as e:
        Config(write(tmp_path, "c.ini", body))
    assert e.value.code == code


def test_ini_device_qbit_key(tmp_path):
    # engine key for the host-resident runner (runner_type IO / DirectIO)
    assert Config(write(tmp_path, "d.ini", "[system]\ntotal_qbit=20\nchunk_qbit=4\n")).device_qbit == 0
    assert Config(write(tmp_path, "e.ini", "[system]\ntotal_qbit=20\nchunk_qbit=4\ndevice_qbit=16\n")).device_qbit == 16
    with pytest.raises(sq.QkError):
        Config(write(tmp_path, "f.ini", "[system]\ntotal_qbit=20\nchunk_qbit=4\ndevice_qbit=21\n"))


def test_ini_missing_file():
    with pytest.raises(sq.QkError) as e:
        Config("/nonexistent/x.ini")
    assert e.value.code == -5


@pytest.mark.parametrize("line,kind,qs,param", [
    ("H 3", 1, [3], 0.0), ("X 0", 2, [0], 0.0), ("Y 1", 3, [1], 0.0), ("Z 2", 4, [2], 0.0),
    ("P 1 0.25", 5, [1], 0.25), ("RX 0 3.141592653589793", 6, [0], np.pi), ("RY 2 -1.5", 7, [2], -1.5),
    ("RZ 3 1e-3", 8, [3], 1e-3), ("SWAP 0 3", 11, [0, 3], 0.0), ("CP  0 1 1.5707963267948966", 12, [0, 1], np.pi / 2),
    ("RZZ 1 2 0.5", 13, [1, 2], 0.5), ("VSWAP_1_1 0 3", 14, [0, 3], 0.0),
    ("VSWAP_2_2 0 1 2 3", 14, [0, 1, 2, 3], 0.0), ("VSWAP_3_3 0 1 2 3 4 5", 14, [0, 1, 2, 3, 4, 5], 0.0),
    ("MPI_VSWAP_2_2 0 1 2 3", 15, [0, 1, 2, 3], 0.0), ("H 1 trailing tokens are ignored", 1, [1], 0.0),
])
def test_parse_line(line, kind, qs, param):
    g = parse_line(line, 6)
    assert g.kind == kind and [g.q[i] for i in range(g.nq)] == qs and g.param == param


@pytest.mark.parametrize("line,code", [
    ("", -2), ("FOO 1", -2), ("U3 0 1 2", -2), ("H", -2), ("RX 0", -2), ("CP 0 1 x", -2),
    ("H 6", -3), ("H -1", -3), ("CP 1 0 0.3", -4), ("CP 1 1 0.3", -4), ("U2 1 0 " + "0 0 " * 16, -4),
    ("VSWAP_2_2 0 1 1 3", -4),
])
def test_parse_errors(line, code):
    with pytest.raises(sq.QkError) as e:
        parse_line(line, 6)
    assert e.value.code == code


def test_subcircuit_format_and_errors():
    c = Circuit.parse("2\nH 0\nCP 0 1 0.5\n1\nVSWAP_2_2 0 1 2 3\n0\n", 1, 4)
    assert c.ngates == 3 and [c.group_sizes[i] for i in range(c.ngroups)] == [2, 1, 0]
    with pytest.raises(sq.QkError):
        Circuit.parse("3\nH 0\n", 1, 4)       # group ends early
    with pytest.raises(sq.QkError):
        Circuit.parse("H 0\n", 1, 4)          # count line expected


def test_circuit_text_round_trip():
    c = circuits.random_u3_cz(6, 3, 7)
    c2 = Circuit.parse(c.to_text(), 0, 6)
    assert c2.ngates == c.ngates
    for a, b in zip(c.gate_list(), c2.gate_list()):
        assert bytes(a) == bytes(b)


def test_gate_matrices_follow_reference_formulas():
    h = gate_matrix(parse_line("H 0", 1))
    assert np.array_equal(h, 0.70710678118 * np.array([[1, 1], [1, -1]]))
    phi = 0.7
    rx = gate_matrix(parse_line(f"RX 0 {phi}", 1))
    assert np.allclose(rx, [[np.cos(phi / 2), 1j * np.sin(-phi / 2)], [1j * np.sin(-phi / 2), np.cos(phi / 2)]])
    rz = gate_matrix(parse_line(f"RZ 0 {phi}", 1))
    assert np.allclose(np.diag(rz), [np.exp(-0.5j * phi), np.exp(0.5j * phi)])
    cp = gate_matrix(parse_line("CP 0 1 3.141592653589793", 2))
    assert cp[3, 3] == complex(np.cos(np.pi), np.sin(np.pi))  # -1 + 1.22e-16 i, as the reference
    # U2: file matrix in basis |a b> with a the MSB -> little-endian (src/circuit.cpp:2811-2819)
    m = np.arange(16).reshape(4, 4) + 1j
    g = make_gate("U2", [0, 1], coeff=m)
    perm = [0, 2, 1, 3]
    assert np.array_equal(gate_matrix(g), m[np.ix_(perm, perm)])
    v = gate_matrix(parse_line("VSWAP_2_2 0 1 2 3", 4))
    assert (v.sum(0) == 1).all() and v[0b0100, 0b0001] == 1 and v[0b1000, 0b0010] == 1


def test_cli_argument_errors():
    r = subprocess.run([CLI, "-x", "y"], capture_output=True, text=True)
    assert r.returncode == 1 and "[Unknown Option]: x" in r.stdout
    r = subprocess.run([CLI, "stray"], capture_output=True, text=True)
    assert r.returncode == 1 and "[Non-option Argument]: stray" in r.stdout


def test_cli_rejects_other_runner_types(tmp_path):
    ini = write(tmp_path, "d.ini", "[system]\ntotal_qbit=4\nchunk_qbit=2\nrunner_type=RDMA\n")
    cir = write(tmp_path, "c.txt", "H 0\n")
    r = subprocess.run([CLI, "-i", ini, "-c", cir], capture_output=True, text=True)
    assert r.returncode == 1 and "runner not found" in r.stderr
