import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
# the test harness's default location of the reference checkout (tests that
# compile against its sources skip where it is absent, e.g. on the GPU box)
os.environ.setdefault("QUOKKA_REFERENCE_DIR", "/root/reference")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def _ensure_built():
    lib = os.path.join(ROOT, "subquokka_dev_b200", "lib", "libquokka_gpu.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-C", os.path.join(ROOT, "subquokka_dev_b200", "csrc"), "-j8"], check=True)
    olib = os.path.join(ROOT, "oracle", "liboracle.so")
    if not os.path.exists(olib):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True)


_ensure_built()


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if gpu_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)
