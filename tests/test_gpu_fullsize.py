"""Parity at the sizes the benchmark measures, against the reference itself.

The 30-qubit, 20-layer random U3 + brick-CZ circuit (seed 2030, the timed
workload) is run by the unmodified reference MEM runner (oracle/_ref,
src/MEM_Runner.cpp:101-134) on the host cores and by this engine on the GPU:
the per-gate complex128 path must match it to 1e-12 in every one of the 2^30
amplitudes, the fused complex128 passes and the complex128 tensor-core blocks
(exact int8 digit products) as well, and the complex64 tensor-core blocks to
1 - F <= 1e-6.  The 30-qubit QFT, written as a
12-qubit-chunk subcircuit file, is run by the reference's subcircuit runner
(src/MEM_Runner.cpp:136-185) and through qk_apply_groups.  The reference's
16 GiB states stay in files and are compared 1 GiB at a time on the GPU.
About five minutes of host time; skipped where the host lacks the memory or
disk, or the reference build is absent.
"""
import math
import os
import shutil

import numpy as np
import pytest

import oracle
from subquokka_dev_b200 import Plan, StateVector, chunk_groups, circuits

pytestmark = pytest.mark.gpu

N = 30
LAYERS = 20
SEED = 2030
TOL_C128 = 1e-12


def _mem_available():
    try:
        for line in open("/proc/meminfo"):
            if line.startswith("MemAvailable:"):
                return int(line.split()[1]) * 1024
    except OSError:
        pass
    return 0


def _skip_reason(tmp):
    if not oracle.have_reference():
        return "reference build (oracle/_ref) absent"
    if _mem_available() < (48 << 30):
        return "host has less than 48 GiB available"
    if shutil.disk_usage(tmp).free < (40 << 30):
        return "less than 40 GB of disk for the reference's states"
    return None


def _file_qbit():
    return max(0, int(math.floor(math.log2(os.cpu_count() or 1))))


def compare(sv, path):
    """(max |delta amp|, 1 - fidelity) of a device state against a raw
    complex128 state file, 1 GiB at a time on the GPU."""
    import torch
    x = sv.as_torch()
    piece = 1 << 26
    dmax, ov, nx, ny = 0.0, 0j, 0.0, 0.0
    for i in range(0, x.numel(), piece):
        r = torch.from_numpy(oracle.read_state_piece(path, i, min(piece, x.numel() - i))).to(x.device)
        g = x[i:i + r.numel()].to(torch.complex128)
        dmax = max(dmax, float((g - r).abs().max()))
        ov += complex(torch.vdot(r, g))
        nx += float(torch.vdot(g, g).real)
        ny += float(torch.vdot(r, r).real)
    return dmax, max(0.0, 1.0 - abs(ov) ** 2 / (nx * ny))


@pytest.fixture(scope="module")
def random30_reference(tmp_path_factory):
    d = tmp_path_factory.mktemp("ref30")
    why = _skip_reason(d)
    if why:
        pytest.skip(why)
    circ = circuits.random_u3_cz(N, LAYERS, SEED)
    out = str(d / "random30.bin")
    _, secs = oracle.run_reference(N, circ.to_text(), 0, chunk_qbit=12, file_qbit=_file_qbit(), out_path=out)
    assert os.path.getsize(out) == 16 << N
    yield circ, out
    os.remove(out)


def test_random30_per_gate_c128_matches_reference(random30_reference):
    circ, ref = random30_reference
    with StateVector(N, "c128") as sv:
        sv.apply(circ)
        sv.synchronize()
        dmax, infid = compare(sv, ref)
    print(f"random-30 per-gate c128 vs reference: max |damp| = {dmax:.3e}, 1 - F = {infid:.3e}")
    assert dmax <= TOL_C128


def test_random30_fused_forms_match_reference(random30_reference):
    circ, ref = random30_reference
    with StateVector(N, "c128") as sv:
        p = Plan(circ, N, "c128")
        p.apply(sv)
        sv.synchronize()
        dmax, _ = compare(sv, ref)
        p.close()
    print(f"random-30 fused c128 passes vs reference: max |damp| = {dmax:.3e}")
    assert dmax <= TOL_C128
    with StateVector(N, "c128") as sv:
        p = Plan(circ, N, "c128", fuse_width=6)
        p.apply(sv)
        sv.synchronize()
        dmax, infid = compare(sv, ref)
        p.close()
    print(f"random-30 c128 int8 tensor-core blocks vs reference: max |damp| = {dmax:.3e}, 1 - F = {infid:.3e}")
    assert dmax <= TOL_C128
    with StateVector(N, "c64") as sv:
        p = Plan(circ, N, "c64", fuse_width=6)
        p.apply(sv)
        sv.synchronize()
        dmax, infid = compare(sv, ref)
        p.close()
    print(f"random-30 c64 tensor-core blocks vs reference: max |damp| = {dmax:.3e}, 1 - F = {infid:.3e}")
    assert infid <= 1e-6
    assert dmax <= 5e-5


def test_qft30_subcircuit_file_matches_reference(tmp_path):
    why = _skip_reason(tmp_path)
    if why:
        pytest.skip(why)
    qft = circuits.qft(N)
    sub = chunk_groups(qft, N, 12)
    out = str(tmp_path / "qft30.bin")
    _, secs = oracle.run_reference(N, sub.to_text(True), 1, chunk_qbit=12, file_qbit=_file_qbit(), out_path=out)
    try:
        with StateVector(N, "c128") as sv:
            sv.apply_groups(sub)
            sv.synchronize()
            dmax, infid = compare(sv, out)
    finally:
        os.remove(out)
    print(f"QFT-30 subcircuit file vs reference subcircuit runner: max |damp| = {dmax:.3e}, 1 - F = {infid:.3e}")
    assert dmax <= TOL_C128
