"""qk_apply_fused_noalloc: the fused-pass path for callers that cannot
allocate device memory (a process whose HBM belongs to a memory pool or to
its own state vectors, or a loop that must not stall on cudaMalloc/cudaFree).

It must give the same state as the existing entry points, call after call,
while keeping its pass programs in the library's fixed device array.  This
file is collected last so that a failure here leaves every other test run.
"""
from ctypes import c_void_p

import numpy as np
import pytest

from subquokka_dev_b200 import QkError, StateVector, _lib, circuits
from subquokka_dev_b200._lib import check

pytestmark = pytest.mark.gpu

TOL_C128 = 1e-12


def noalloc(sv, circ):
    check(_lib.load().qk_apply_fused_noalloc(c_void_p(sv.device_ptr), sv.nqubits, sv.dtype, circ.gates,
                                             circ.ngates, None))


def existing(n, circ, init):
    with StateVector(n) as sv:
        sv.upload(init)
        sv.apply(circ)          # qk_apply_gates, the per-gate entry point
        return sv.download()


def test_noalloc_matches_existing_entry_point_two_calls_in_a_row():
    n = 16
    first, second = circuits.random_u3_cz(n, 8, 41), circuits.hea(n, 3, 42)[0]
    init = circuits.random_state(n, 43)
    with StateVector(n) as sv:
        sv.upload(init)
        noalloc(sv, first)
        out1 = sv.download()
        # second call, different programs, same shared device array
        sv.upload(init)
        noalloc(sv, second)
        out2 = sv.download()
    assert np.abs(out1 - existing(n, first, init)).max() <= TOL_C128
    assert np.abs(out2 - existing(n, second, init)).max() <= TOL_C128


def test_noalloc_rejects_circuits_beyond_the_array():
    n = 12
    big = circuits.random_u3_cz(n, 1200, 44)   # > 1 MiB of pass programs
    with StateVector(n) as sv:
        with pytest.raises(QkError) as e:
            noalloc(sv, big)
    assert e.value.code == -1 and "holds at most" in str(e.value)
