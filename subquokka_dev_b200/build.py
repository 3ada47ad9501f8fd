"""In-tree build of the engine: ``python -m subquokka_dev_b200.build``.

Compiles libquokka_gpu.so and the quokka CLI for sm_100a (csrc/Makefile) into
subquokka_dev_b200/lib and subquokka_dev_b200/bin, so they travel with the
source tree.
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG_DIR = os.path.dirname(os.path.abspath(__file__))


def build(jobs: int = 8) -> None:
    subprocess.run(["make", "-C", os.path.join(PKG_DIR, "csrc"), f"-j{jobs}"], check=True)


if __name__ == "__main__":
    build(int(sys.argv[1]) if len(sys.argv) > 1 else 8)
