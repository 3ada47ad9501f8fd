"""Host-resident states (qk_hsv_*): the state in pinned host memory, the
gates on the GPU chunk by chunk.  Against the FP64 oracle and the in-HBM
per-gate path, for chunks much smaller than the state (many chunks per
segment, several segments, gathers with strides)."""
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
