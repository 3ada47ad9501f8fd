"""CPU checks of the planner, built from the host sources with g++:
- tests/rewrite_check.cpp: the op-list rewrites the planners apply before
  compiling pass programs (one-qubit merges, folds into two-qubit and
  conditioned ops, gradient hoisting and pairing, ASAP order, VSWAP
  renaming) keep the states and gradients a list computes;
- tests/plan_check.cpp: forward and adjoint fused plans, run by an emulator
  of the pass programs, give the states and gradients of the dense
  simulation of their gate lists."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "subquokka_dev_b200", "csrc")


def build_and_run(tmp_path, main, sources):
    # built with AddressSanitizer and UndefinedBehaviorSanitizer: the host
    # planner code also runs free of memory errors, leaks and undefined
    # behaviour on these inputs
    exe = tmp_path / main.replace(".cpp", "")
    cmd = ["g++", "-O1", "-g", "-std=c++17", "-fsanitize=address,undefined", "-fno-omit-frame-pointer",
           "-I", os.path.join(ROOT, "include"), "-I", CSRC, "-I", os.path.join(ROOT, "tests"),
           os.path.join(ROOT, "tests", main)]
    cmd += [os.path.join(CSRC, f) for f in sources] + ["-o", str(exe)]
    build = subprocess.run(cmd, capture_output=True, text=True)
    assert build.returncode == 0, build.stderr
    env = dict(os.environ, UBSAN_OPTIONS="halt_on_error=1:print_stacktrace=1", ASAN_OPTIONS="detect_leaks=1")
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout + r.stderr


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ absent")
def test_rewrites_keep_states_and_gradients(tmp_path):
    build_and_run(tmp_path, "rewrite_check.cpp", ["qk_rewrite.cpp", "qk_parse.cpp"])


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ absent")
def test_plans_compute_the_circuit(tmp_path):
    build_and_run(tmp_path, "plan_check.cpp", ["qk_plan.cpp", "qk_rewrite.cpp", "qk_parse.cpp", "qk_dense_host.cpp"])
