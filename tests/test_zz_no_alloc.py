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
TOL_C64 = 2e-6   # complex64 storage, as in the other complex64 tests
SCRATCH_BYTES = 1 << 20   # QK_NOALLOC_SCRATCH_BYTES
QK_ERR_UNSUPPORTED = -8


def noalloc(sv, circ, stream=None):
    check(_lib.load().qk_apply_fused_noalloc(c_void_p(sv.device_ptr), sv.nqubits, sv.dtype, circ.gates,
                                             circ.ngates, c_void_p(stream or 0)))


def existing(n, circ, init, dtype="c128"):
    with StateVector(n, dtype) as sv:
        sv.upload(init)
        sv.apply(circ)          # qk_apply_gates, the per-gate entry point
        return sv.download()


@pytest.mark.parametrize("dtype,tol", [("c128", TOL_C128), ("c64", TOL_C64)])
def test_noalloc_matches_existing_entry_point_two_calls_in_a_row(dtype, tol):
    n = 16
    first, second = circuits.random_u3_cz(n, 8, 41), circuits.hea(n, 3, 42)[0]
    init = circuits.random_state(n, 43)
    with StateVector(n, dtype) as sv:
        sv.upload(init)
        noalloc(sv, first)
        out1 = sv.download()
        # second call, different programs, same shared device array
        sv.upload(init)
        noalloc(sv, second)
        out2 = sv.download()
    assert np.abs(out1 - existing(n, first, init, dtype)).max() <= tol
    assert np.abs(out2 - existing(n, second, init, dtype)).max() <= tol


def test_noalloc_two_circuits_back_to_back_on_one_stream():
    """Two calls on one created stream, no host synchronisation between them:
    the second call's programs overwrite the first's only after the first
    call's passes ran (stream order)."""
    import torch
    n = 15
    a, b = circuits.random_u3_cz(n, 6, 51), circuits.qft(n)
    init = circuits.random_state(n, 52)
    st = torch.cuda.Stream()
    with StateVector(n) as s1, StateVector(n) as s2:
        s1.set_stream(st.cuda_stream)
        s2.set_stream(st.cuda_stream)
        s1.upload(init)
        s2.upload(init)
        noalloc(s1, a, st.cuda_stream)
        noalloc(s2, b, st.cuda_stream)
        st.synchronize()
        o1, o2 = s1.download(), s2.download()
    assert np.abs(o1 - existing(n, a, init)).max() <= TOL_C128
    assert np.abs(o2 - existing(n, b, init)).max() <= TOL_C128


def test_noalloc_rejects_circuits_beyond_the_array():
    n = 12
    big = circuits.random_u3_cz(n, 5000, 44)   # several MiB of pass programs and coefficients
    # at least one 16-byte program op per CZ pair of a layer, each folded CZ a
    # 4x4 complex128 matrix of 256 bytes: far above the 1 MiB array
    assert (n // 2) * 5000 * (16 + 256) > 4 * SCRATCH_BYTES
    with StateVector(n) as sv:
        with pytest.raises(QkError) as e:
            noalloc(sv, big)
    assert e.value.code == -1 and "holds at most" in str(e.value)


def test_noalloc_refuses_a_capturing_stream():
    """Its copies come from host memory freed on return, and it waits for them:
    neither can be recorded into a graph, so the call is refused."""
    import torch
    n = 10
    circ = circuits.random_u3_cz(n, 2, 61)
    with StateVector(n) as sv:
        noalloc(sv, circ)   # set-up on this device, outside any capture
        st = torch.cuda.Stream()
        g = torch.cuda.CUDAGraph()
        code = None
        with torch.cuda.stream(st):
            g.capture_begin()
            try:
                noalloc(sv, circ, st.cuda_stream)
            except QkError as e:
                code = e.code
            finally:
                g.capture_end()
        del g
    assert code == QK_ERR_UNSUPPORTED
