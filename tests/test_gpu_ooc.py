"""Host-resident states (qk_hsv_*): the state in pinned host memory, the
gates on the GPU chunk by chunk.  Against the FP64 oracle and the in-HBM
per-gate path, for chunks much smaller than the state (many chunks per
segment, several segments, gathers with strides)."""
import os
import subprocess

import numpy as np
import pytest

import oracle
from subquokka_dev_b200 import HostStateVector, StateVector, circuits, ooc_segments
from test_ooc_host import random_mixed

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind,n,L", [("random_u3_cz", 18, 14), ("random_u3_cz", 18, 12), ("qft", 16, 12),
                                      ("mixed", 15, 12), ("random_u3_cz", 16, 16)])
def test_host_state_matches_oracle(kind, n, L):
    circ = (circuits.random_u3_cz(n, 8, 21) if kind == "random_u3_cz" else circuits.qft(n) if kind == "qft"
            else random_mixed(n, 200, 22))
    init = circuits.random_state(n, 23)
    with HostStateVector(n, L, "c128") as h:
        h.view()[:] = init
        h.apply(circ)
        out = h.view().copy()
        st = h.stats()
    assert st["segments"] == len(ooc_segments(circ, n, L)) and st["device_ms"] > 0
    ref = oracle.apply_circuit(init, n, circ)
    assert np.abs(out - ref).max() <= 1e-12


def test_host_state_complex64_and_two_calls():
    n, L = 17, 13
    a, b = circuits.random_u3_cz(n, 5, 31), circuits.qft(n)
    with HostStateVector(n, L, "c64") as h:
        h.apply(a)
        h.apply(b)                      # continues from the first call's state
        out = h.view().astype(np.complex128)
    with StateVector(n, "c128") as sv:
        sv.apply(a)
        sv.apply(b)
        ref = sv.download()
    assert np.abs(out - ref).max() <= 2e-6


def test_host_state_reset_and_empty_circuit():
    from subquokka_dev_b200 import Circuit
    with HostStateVector(12, 10) as h:
        h.apply(circuits.qft(12))
        h.reset()
        h.apply(Circuit([]))
        v = h.view()
        assert v[0] == 1 and np.count_nonzero(v) == 1


CLI = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "subquokka_dev_b200", "bin",
                   "quokka")


@pytest.mark.parametrize("name,dq,precision,tol", [("qft12", 8, "c128", 1e-12), ("sub12", 9, "c128", 1e-12),
                                                   ("rand10", 7, "c128", 1e-12), ("qft21", 17, "c128", 1e-12),
                                                   ("qft12", 9, "c64", 2e-6)])
def test_cli_io_runner_on_host_state(tmp_path, name, dq, precision, tol):
    """runner_type=IO: the reference's out-of-core runner's slot, here the
    state in host memory and 2^device_qbit-amplitude chunks on the GPU; the
    reference's golden final states (flat and subcircuit files)."""
    import golden_util as gu
    rec = gu.load(name)
    gu.initial_state(rec).astype(np.complex128).tofile(tmp_path / "init.bin")
    ini = tmp_path / "io.ini"
    ini.write_text(f"[system]\ntotal_qbit={rec['n']}\nfile_qbit=0\nchunk_qbit=4\nrunner_type=IO\n"
                   f"is_subcircuit={rec['is_subcircuit']}\ninit_file={tmp_path}/init.bin\ndevice_qbit={dq}\n"
                   f"precision={precision}\ndump_file={tmp_path}/state.bin\ndump_format=bin\n")
    (tmp_path / "c.txt").write_text(rec["circuit"])
    r = subprocess.run([CLI, "-i", str(ini), "-c", str(tmp_path / "c.txt")], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    assert "IO Mode" in r.stdout
    assert gu.compare(rec, np.fromfile(tmp_path / "state.bin", dtype=np.complex128)) <= tol
