"""B200-native state-vector engine for the SubQuokka simulator's in-memory path.

The engine keeps the 2^N-amplitude state resident in HBM and applies the
gates of the reference's circuit.txt format with hand-written sm_100a
kernels behind a C ABI (include/quokka_gpu.h, libquokka_gpu.so).  This package
is the Python side of that ABI: ctypes bindings (_lib), the runner mirror
(engine) and the seeded workloads (circuits).
"""
from .engine import (Batch, Circuit, Config, GateGraph, HostStateVector, Plan, Simulator, StateVector, adjoint_grad, apply_gates_dev,
                     chunk_groups, expval, gate_line, gate_matrix, last_sweep, make_gate, ooc_segments, parse_line, pauli_terms,
                     zz_x_hamiltonian)
from ._lib import QkError, load as load_library

__all__ = ["Batch", "Circuit", "Config", "GateGraph", "HostStateVector", "Plan", "Simulator", "StateVector", "adjoint_grad", "apply_gates_dev",
           "chunk_groups", "expval", "last_sweep", "ooc_segments",
           "gate_line", "gate_matrix", "make_gate", "parse_line", "pauli_terms", "zz_x_hamiltonian", "QkError",
           "load_library"]
