"""The op-list rewrites the planners apply before compiling pass programs
(one-qubit merges, folds into two-qubit and conditioned ops, gradient
hoisting and pairing, ASAP order, VSWAP renaming) keep the states and
gradients a list computes: tests/rewrite_check.cpp runs random lists and
their rewritten forms on small dense states on the CPU."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "subquokka_dev_b200", "csrc")


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ absent")
def test_rewrites_keep_states_and_gradients(tmp_path):
    exe = tmp_path / "rewrite_check"
    cmd = ["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), "-I", CSRC,
           os.path.join(ROOT, "tests", "rewrite_check.cpp"), os.path.join(CSRC, "qk_rewrite.cpp"),
           os.path.join(CSRC, "qk_parse.cpp"), "-o", str(exe)]
    build = subprocess.run(cmd, capture_output=True, text=True)
    assert build.returncode == 0, build.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout + r.stderr
