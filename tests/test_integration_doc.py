"""The reference-side GPU_Runner that INTEGRATION.md shows is the committed
binding (subquokka_dev_b200/runner/GPU_Runner.hpp, .cpp), and it builds into
the reference: oracle/_ref/Quokka_gpu is the reference's CLI with a copy of
simulator.cpp whose GPU stub gpu_slot.py replaces.  On the CPU: the document
matches the files, the patch applies to the reference's source, and the
patched binary still runs the reference's own MEM runner unchanged.  (The GPU
runs of the same binary are tests/test_gpu_reference_runner.py.)"""
import os
import re
import shutil
import subprocess
import sys

import numpy as np
import pytest

import golden_util as gu
import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RUNNER = os.path.join(ROOT, "subquokka_dev_b200", "runner")
EXE = os.path.join(ROOT, "oracle", "_ref", "Quokka_gpu")


def test_integration_doc_shows_the_committed_gpu_runner():
    md = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    blocks = re.findall(r"```cpp\n(.*?)```", md, re.S)
    hpp = open(os.path.join(RUNNER, "GPU_Runner.hpp")).read()
    assert hpp in blocks, "INTEGRATION.md must show GPU_Runner.hpp as committed"
    assert "class GPU_Runner : public Simulator::circuitRunner" in hpp


@pytest.mark.skipif(not oracle.have_reference_source(), reason="reference sources absent")
def test_gpu_slot_patch_applies_to_the_reference_source():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import gpu_slot
    src = open(os.path.join(oracle.REF_SOURCE, "src", "simulator.cpp")).read()
    out = gpu_slot.patch(src)
    assert "Runner = new GPU_Runner(ini);" in out
    assert out.count('env.runner_type != "GPU"') == 2
    assert "GPU runner not found" not in out


@pytest.mark.skipif(not os.path.exists(EXE) or shutil.which("g++") is None, reason="oracle/_ref/Quokka_gpu not built")
def test_patched_reference_still_runs_its_mem_runner(tmp_path):
    rec = gu.load("rand10")
    n = rec["n"]
    (tmp_path / "x.ini").write_text(f"[system]\ntotal_qbit={n}\nfile_qbit={int(rec['file_qbit'])}\n"
                                    f"chunk_qbit={int(rec['chunk_qbit'])}\nrunner_type=MEM\nis_subcircuit=0\n"
                                    "dump_file=mem.txt\nMPI_testing=1\n")
    (tmp_path / "c.txt").write_text(rec["circuit"])
    r = subprocess.run([EXE, "-i", "x.ini", "-c", "c.txt"], capture_output=True, text=True, cwd=tmp_path, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "MEM Mode" in r.stdout
    vals = np.loadtxt(tmp_path / "mem0.txt")
    assert np.abs(vals[0::2] + 1j * vals[1::2] - rec["final"]).max() <= 1e-11
