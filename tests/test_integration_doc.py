"""The reference-side GPU_Runner that INTEGRATION.md shows (section 1) is
real code: it compiles against the reference's own headers (simulator.hpp,
with the oracle's stand-in mpi.h), and links with the reference's objects
(oracle/_ref) and libquokka_gpu.so into a program that loads the library.
Runs where the reference sources and their build are present."""
import os
import re
import shutil
import subprocess

import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
OBJ = os.path.join(ROOT, "oracle", "_ref", "obj")

pytestmark = pytest.mark.skipif(
    shutil.which("g++") is None or not oracle.have_reference_source() or not os.path.isdir(OBJ),
    reason="reference sources or their build (oracle/_ref) absent")


def test_documented_gpu_runner_builds_into_the_reference(tmp_path):
    md = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    runner = re.findall(r"```cpp\n(.*?)```", md, re.S)[0]
    assert "class GPU_Runner : public Simulator::circuitRunner" in runner
    (tmp_path / "gpu_runner.cpp").write_text(
        runner + "\nvoid GPU_Runner::run(std::vector<Gate *> &) {}\n"
                 "void GPU_Runner::run(std::vector<std::vector<Gate *>> &) {}\n"
                 "Simulator::circuitRunner *make_gpu_runner() { return new GPU_Runner(); }\n")
    (tmp_path / "main.cpp").write_text(
        '#include <cstdio>\n#include "simulator.hpp"\n#include "quokka_gpu.h"\n'
        "Simulator::circuitRunner *make_gpu_runner();\n"
        'int main() { std::printf("abi %d\\n", qk_abi_version()); return make_gpu_runner ? 0 : 1; }\n')
    objs = [os.path.join(OBJ, f) for f in sorted(os.listdir(OBJ)) if f.endswith(".o") and f != "main.o"]
    lib = os.path.join(ROOT, "subquokka_dev_b200", "lib")
    exe = tmp_path / "linked"
    cmd = ["g++", "-std=c++17", "-fopenmp", "-I", os.path.join(oracle.REF_SOURCE, "src"), "-I",
           os.path.join(ROOT, "oracle", "stub"), "-I", os.path.join(ROOT, "include"),
           str(tmp_path / "gpu_runner.cpp"), str(tmp_path / "main.cpp")] + objs + \
          ["-L", lib, "-lquokka_gpu", "-Wl,-rpath," + lib, "-o", str(exe)]
    build = subprocess.run(cmd, capture_output=True, text=True)
    assert build.returncode == 0, build.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and r.stdout.strip() == "abi 2", r.stdout + r.stderr
