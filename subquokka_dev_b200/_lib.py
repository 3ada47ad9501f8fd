"""ctypes binding of libquokka_gpu.so (the C ABI declared in include/quokka_gpu.h).

The library is built in-tree (``python -m subquokka_dev_b200.build``) into
``subquokka_dev_b200/lib``.  Loading fails loudly when it is missing: there is
no CPU fallback anywhere in the engine.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char, c_char_p, c_double, c_int, c_int32, c_size_t, c_void_p

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "lib", "libquokka_gpu.so")

QK_MAX_TARGETS = 12
QK_C128, QK_C64 = 0, 1

# qk_gate_kind
ABI_VERSION = 3   # QK_ABI_VERSION of include/quokka_gpu.h that QkGate / QkConfig below mirror

GATE_KINDS = {
    "H": 1, "X": 2, "Y": 3, "Z": 4, "P": 5, "RX": 6, "RY": 7, "RZ": 8,
    "U1": 9, "U2": 10, "SWAP": 11, "CP": 12, "RZZ": 13, "VSWAP": 14, "MPI_VSWAP": 15,
}
KIND_NAMES = {v: k for k, v in GATE_KINDS.items()}

STATUS = {
    0: "QK_OK", -1: "QK_ERR_ARG", -2: "QK_ERR_PARSE", -3: "QK_ERR_QUBIT", -4: "QK_ERR_ORDER",
    -5: "QK_ERR_IO", -6: "QK_ERR_CUDA", -7: "QK_ERR_OOM", -8: "QK_ERR_UNSUPPORTED", -9: "QK_ERR_NOT_BUILT",
}


class QkGate(ctypes.Structure):
    _fields_ = [
        ("kind", c_int32),
        ("nq", c_int32),
        ("q", c_int32 * QK_MAX_TARGETS),
        ("param", c_double),
        ("coeff", c_double * 32),
    ]


class QkConfig(ctypes.Structure):
    _fields_ = [
        ("total_qbit", c_int32),
        ("mpi_qbit", c_int32),
        ("file_qbit", c_int32),
        ("chunk_qbit", c_int32),
        ("is_subcircuit", c_int32),
        ("MPI_testing", c_int32),
        ("MPI_buffe_size", c_int32),
        ("precision", c_int32),
        ("fuse_width", c_int32),
        ("dump_binary", c_int32),
        ("runner_type", c_char * 32),
        ("dump_file", c_char * 256),
        ("init_file", c_char * 256),
        ("device_qbit", c_int32),
    ]


class QkPlanOpts(ctypes.Structure):
    _fields_ = [("dtype", c_int32), ("tile_bits", c_int32), ("reg_bits", c_int32), ("fuse_width", c_int32),
                ("reserved", c_int32 * 4)]


class QkPauliTerm(ctypes.Structure):
    _fields_ = [("coeff", c_double), ("x_mask", ctypes.c_uint64), ("z_mask", ctypes.c_uint64)]


class QkBatchOpts(ctypes.Structure):
    _fields_ = [("dtype", c_int32), ("autotune", c_int32), ("tile_bits", c_int32), ("reg_bits", c_int32),
                ("adj_tile_bits", c_int32), ("adj_reg_bits", c_int32), ("reserved", c_int32 * 2)]


class QkError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, code: int, message: str):
        super().__init__(f"{STATUS.get(code, code)}: {message}")
        self.code = code


# name -> (restype, argtypes); every symbol include/quokka_gpu.h declares.
PROTOTYPES = {
    "qk_last_error": (c_char_p, []),
    "qk_abi_version": (c_int, []),
    "qk_config_load": (c_int, [c_char_p, POINTER(QkConfig)]),
    "qk_gate_parse_line": (c_int, [c_char_p, c_int, POINTER(QkGate)]),
    "qk_circuit_load": (c_int, [c_char_p, c_int, c_int, POINTER(c_void_p)]),
    "qk_circuit_parse": (c_int, [c_char_p, c_int, c_int, POINTER(c_void_p)]),
    "qk_circuit_num_gates": (c_size_t, [c_void_p]),
    "qk_circuit_gates": (POINTER(QkGate), [c_void_p]),
    "qk_circuit_num_groups": (c_size_t, [c_void_p]),
    "qk_circuit_group_sizes": (POINTER(c_int32), [c_void_p]),
    "qk_circuit_destroy": (None, [c_void_p]),
    "qk_gate_matrix": (c_int, [POINTER(QkGate), POINTER(c_double), POINTER(c_int)]),
    "qk_circuit_chunk_groups": (c_int, [POINTER(QkGate), c_size_t, c_int, c_int, POINTER(c_void_p)]),
    "qk_circuit_write": (c_int, [c_void_p, c_int, c_char_p]),
    "qk_sv_create": (c_int, [c_int, c_int, POINTER(c_void_p)]),
    "qk_sv_destroy": (None, [c_void_p]),
    "qk_sv_reset": (c_int, [c_void_p]),
    "qk_sv_upload": (c_int, [c_void_p, POINTER(c_double)]),
    "qk_sv_download": (c_int, [c_void_p, POINTER(c_double)]),
    "qk_sv_save": (c_int, [c_void_p, c_char_p]),
    "qk_sv_load": (c_int, [c_void_p, c_char_p]),
    "qk_sv_info": (c_int, [c_void_p, POINTER(c_int), POINTER(c_int), POINTER(c_void_p), POINTER(c_size_t)]),
    "qk_sv_set_stream": (c_int, [c_void_p, c_void_p]),
    "qk_sv_synchronize": (c_int, [c_void_p]),
    "qk_sv_release_workspace": (c_int, [c_void_p]),
    "qk_sv_last_sweep": (c_int, [c_void_p, POINTER(c_double), POINTER(c_double), POINTER(c_int), POINTER(c_int)]),
    "qk_batch_timing": (c_int, [c_void_p, POINTER(c_double), POINTER(c_double)]),
    "qk_hsv_create": (c_int, [c_int, c_int, c_int, POINTER(c_void_p)]),
    "qk_hsv_reset": (c_int, [c_void_p]),
    "qk_hsv_data": (c_void_p, [c_void_p]),
    "qk_hsv_apply_gates": (c_int, [c_void_p, POINTER(QkGate), c_size_t]),
    "qk_hsv_stats": (c_int, [c_void_p, POINTER(c_int), POINTER(c_double), POINTER(c_double)]),
    "qk_hsv_destroy": (None, [c_void_p]),
    "qk_ooc_segments": (c_int, [POINTER(QkGate), c_size_t, c_int, c_int, POINTER(ctypes.c_uint64), POINTER(c_int32),
                                POINTER(c_int32), c_size_t, POINTER(c_size_t)]),
    "qk_apply_gates": (c_int, [c_void_p, POINTER(QkGate), c_size_t]),
    "qk_graph_create": (c_int, [c_void_p, POINTER(QkGate), c_size_t, POINTER(c_void_p)]),
    "qk_graph_launch": (c_int, [c_void_p]),
    "qk_graph_destroy": (None, [c_void_p]),
    "qk_apply_groups": (c_int, [c_void_p, POINTER(QkGate), POINTER(c_int32), c_size_t]),
    "qk_apply_gates_dev": (c_int, [c_void_p, c_int, c_int, POINTER(QkGate), c_size_t, c_void_p]),
    "qk_apply_gates_timed": (c_int, [c_void_p, POINTER(QkGate), c_size_t, POINTER(ctypes.c_float)]),
    "qk_plan_create": (c_int, [POINTER(QkGate), c_size_t, c_int, POINTER(QkPlanOpts), POINTER(c_void_p)]),
    "qk_plan_create_groups": (c_int, [POINTER(QkGate), POINTER(c_int32), c_size_t, c_int, POINTER(QkPlanOpts),
                                      POINTER(c_void_p)]),
    "qk_plan_stats": (c_int, [c_void_p, POINTER(c_size_t), POINTER(c_size_t), POINTER(c_size_t)]),
    "qk_plan_apply": (c_int, [c_void_p, c_void_p]),
    "qk_plan_dense_block": (c_int, [c_void_p, c_size_t, POINTER(c_int32), POINTER(c_double), POINTER(c_int)]),
    "qk_plan_destroy": (None, [c_void_p]),
    "qk_apply_fused_noalloc": (c_int, [c_void_p, c_int, c_int, POINTER(QkGate), c_size_t, c_void_p]),
    "qk_expval_pauli": (c_int, [c_void_p, POINTER(QkPauliTerm), c_size_t, POINTER(c_double)]),
    "qk_adjoint_grad": (c_int, [c_void_p, POINTER(QkGate), c_size_t, POINTER(c_int32), c_size_t, POINTER(QkPauliTerm),
                                c_size_t, c_int, POINTER(c_double), POINTER(c_double), POINTER(c_double)]),
    "qk_adjoint_grad_fused": (c_int, [c_void_p, POINTER(QkGate), c_size_t, POINTER(c_int32), c_size_t,
                                      POINTER(QkPauliTerm), c_size_t, c_int, POINTER(c_double), POINTER(c_double),
                                      POINTER(c_double)]),
    "qk_batch_create": (c_int, [c_int, POINTER(c_int32), POINTER(QkGate), POINTER(c_size_t), POINTER(c_int32),
                                POINTER(c_size_t), POINTER(QkPauliTerm), POINTER(c_size_t), POINTER(QkBatchOpts),
                                POINTER(c_void_p)]),
    "qk_batch_run": (c_int, [c_void_p, POINTER(c_double), POINTER(c_double), POINTER(c_double)]),
    "qk_batch_set_params": (c_int, [c_void_p, POINTER(c_double)]),
    "qk_batch_stats": (c_int, [c_void_p, POINTER(c_int), POINTER(c_int), POINTER(c_int), POINTER(c_int),
                               POINTER(c_int), POINTER(c_int)]),
    "qk_batch_destroy": (None, [c_void_p]),
    "qk_run": (c_int, [POINTER(QkConfig), c_void_p, c_void_p, POINTER(c_double)]),
}

_lib = None


def load() -> ctypes.CDLL:
    """Load (once) and return the engine library; raise if it is not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with `python -m subquokka_dev_b200.build` "
            "(the engine has no CPU fallback)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.qk_abi_version() != ABI_VERSION:   # the structures above must match the library's
        raise RuntimeError(f"{LIB_PATH} has ABI version {lib.qk_abi_version()}, these bindings {ABI_VERSION}: "
                           "rebuild it with `python -m subquokka_dev_b200.build`")
    _lib = lib
    return lib


def last_error() -> str:
    return load().qk_last_error().decode(errors="replace")


def check(code: int) -> None:
    if code != 0:
        raise QkError(code, last_error())
