"""ORACLE -- test infrastructure only (tests/, __graft_entry__.smoke(), the
CPU-baseline leg of bench.py).  The product never imports this package.

ctypes access to the C restatement (qk_oracle.c -> liboracle.so) and to the
unmodified reference build (_ref/quokka_ref, made by ``make -C oracle ref``
from the reference's own sources).
"""
from __future__ import annotations

import ctypes
import os
import re
import subprocess
import tempfile
from ctypes import POINTER, c_double, c_int, c_size_t

import numpy as np

ORACLE_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(ORACLE_DIR, "liboracle.so")
REF_DRIVER = os.path.join(ORACLE_DIR, "_ref", "quokka_ref")
# the reference checkout whose sources `make ref` compiles; only set where
# those sources exist (the build and test harnesses pass it in)
REF_SOURCE = os.environ.get("QUOKKA_REFERENCE_DIR", "")

_lib = None


def have_reference_source(ref_dir: str | None = None) -> bool:
    d = REF_SOURCE if ref_dir is None else ref_dir
    return bool(d) and os.path.isdir(os.path.join(d, "src"))


def build(with_reference: bool | None = None, ref_dir: str | None = None) -> None:
    """Compile the C restatement and, when the reference sources are present
    (ref_dir, else $QUOKKA_REFERENCE_DIR), the reference itself (oracle/_ref)."""
    d = REF_SOURCE if ref_dir is None else ref_dir
    subprocess.run(["make", "-C", ORACLE_DIR], check=True)
    if with_reference is None:
        with_reference = have_reference_source(d)
    if with_reference:
        subprocess.run(["make", "-C", ORACLE_DIR, "ref", "-j8", f"REF={d}"], check=True)
        # the reference CLI with the engine in its GPU slot (needs the built library)
        if os.path.exists(os.path.join(ORACLE_DIR, "..", "subquokka_dev_b200", "lib", "libquokka_gpu.so")):
            subprocess.run(["make", "-C", ORACLE_DIR, "ref-gpu", f"REF={d}"], check=True)


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build(with_reference=False)
        from subquokka_dev_b200._lib import QkGate
        lib = ctypes.CDLL(LIB_PATH)
        lib.qko_apply.argtypes = [POINTER(c_double), c_int, POINTER(QkGate)]
        lib.qko_apply.restype = c_int
        lib.qko_apply_list.argtypes = [POINTER(c_double), c_int, POINTER(QkGate), c_size_t]
        lib.qko_apply_list.restype = c_int
        lib.qko_expval_zz_x.argtypes = [POINTER(c_double), c_int, POINTER(c_double), POINTER(c_double)]
        lib.qko_expval_zz_x.restype = c_double
        lib.qko_adjoint_grad.argtypes = [POINTER(c_double), c_int, POINTER(QkGate), c_size_t, POINTER(c_int), c_size_t,
                                         ctypes.c_void_p, c_size_t, POINTER(c_double), POINTER(c_double)]
        lib.qko_adjoint_grad.restype = c_int
        _lib = lib
    return _lib


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(POINTER(c_double))


def apply_circuit(state: np.ndarray, n: int, circuit) -> np.ndarray:
    """Apply a circuit (subquokka_dev_b200.Circuit) to a copy of state; FP64."""
    s = np.array(state, dtype=np.complex128, copy=True)
    rc = load().qko_apply_list(_dptr(s), n, circuit.gates, circuit.ngates)
    if rc:
        raise RuntimeError("oracle: unknown gate")
    return s


def expval_zz_x(state: np.ndarray, n: int, J, h) -> float:
    s = np.ascontiguousarray(state, dtype=np.complex128)
    J = np.ascontiguousarray(J, dtype=np.float64)
    h = np.ascontiguousarray(h, dtype=np.float64)
    return load().qko_expval_zz_x(_dptr(s), n, _dptr(J), _dptr(h))


def have_reference() -> bool:
    return os.path.exists(REF_DRIVER)


def run_reference(n: int, circuit_text: str, is_subcircuit: int, init: np.ndarray | None = None,
                  chunk_qbit: int = 12, file_qbit: int = 0, threads: int | None = None,
                  out_path: str | None = None):
    """Run the unmodified reference MEM runner; returns (final state, runner
    seconds).  With out_path the final state stays in that file (raw
    complex128) and None is returned in its place: large states are then read
    piece by piece (read_state_piece) instead of as one host array."""
    chunk = min(chunk_qbit, n - file_qbit)
    with tempfile.TemporaryDirectory() as d:
        ini = os.path.join(d, "x.ini")
        with open(ini, "w") as f:
            f.write(f"[system]\ntotal_qbit={n}\nfile_qbit={file_qbit}\nchunk_qbit={chunk}\n"
                    f"runner_type=MEM\nis_subcircuit={int(is_subcircuit)}\n")
        cir = os.path.join(d, "c.txt")
        with open(cir, "w") as f:
            f.write(circuit_text)
        out = out_path or os.path.join(d, "out.bin")
        cmd = [REF_DRIVER, "-i", ini, "-c", cir, "-o", out]
        if init is not None:
            ip = os.path.join(d, "init.bin")
            np.ascontiguousarray(init, dtype=np.complex128).tofile(ip)
            cmd += ["-s", ip]
        env = dict(os.environ)
        if threads:
            env["OMP_NUM_THREADS"] = str(threads)
        r = subprocess.run(cmd, capture_output=True, text=True, env=env, check=True)
        m = re.search(r"^([0-9.eE+-]+)s$", r.stdout, re.M)
        secs = float(m.group(1)) if m else float("nan")
        if out_path:
            return None, secs
        return np.fromfile(out, dtype=np.complex128), secs


def read_state_piece(path: str, first: int, count: int) -> np.ndarray:
    """Amplitudes [first, first + count) of a raw complex128 state file."""
    return np.fromfile(path, dtype=np.complex128, count=count, offset=16 * first)


def pauli_expval(state: np.ndarray, n: int, terms) -> float:
    """<psi|H|psi> for terms (coeff, x_mask, z_mask), H = sum coeff i^popcount(x&z) X^x Z^z; FP64 numpy."""
    psi = np.asarray(state, dtype=np.complex128)
    idx = np.arange(1 << n, dtype=np.uint64)
    total = 0.0
    for c, x, z in terms:
        src = idx ^ np.uint64(x)
        sign = 1.0 - 2.0 * (np.bitwise_count(src & np.uint64(z)) & 1)
        phase = 1j ** (bin(int(x) & int(z)).count("1") % 4)
        # (P psi)[j] = phase * sign(src) * psi[src] with src = j ^ x
        pj = phase * sign * psi[src.astype(np.int64)]
        total += float(c) * float(np.vdot(psi, pj).real)
    return total


def param_shift_grad(pc, params: np.ndarray, terms) -> np.ndarray:
    """Parameter-shift gradient of <H> for a torch_shim.ParamCircuit whose
    trainable gates are RX/RY/RZ (exp(-i theta P / 2)): per occurrence,
    (E(theta + pi/2) - E(theta - pi/2)) / 2; FP64 on the CPU oracle."""
    n = pc.n
    z0 = np.zeros(1 << n, np.complex128)
    z0[0] = 1

    def energy(vals):
        circ, _ = pc.bind(vals)
        return pauli_expval(apply_circuit(z0, n, circ), n, terms)

    grad = np.zeros(pc.nparams)
    for k, (_, _, _, p, _) in enumerate(pc.ops):
        if p < 0:
            continue
        # shift only this occurrence: bind, then edit the gate's angle
        for sgn in (+1, -1):
            circ, _ = pc.bind(params)
            g = circ.gates[k]
            g.param = g.param + sgn * np.pi / 2
            e = pauli_expval(apply_circuit(z0, n, circ), n, terms)
            grad[p] += sgn * e / 2
    return grad


class _Term(ctypes.Structure):
    _fields_ = [("coeff", c_double), ("x", ctypes.c_ulonglong), ("z", ctypes.c_ulonglong)]


def adjoint_grad(state: np.ndarray, n: int, circuit, pidx, nparams: int, terms):
    """FP64 CPU adjoint restatement: (<H>, gradient) after circuit on state."""
    s = np.array(state, dtype=np.complex128, copy=True)
    p = np.ascontiguousarray(pidx, dtype=np.int32)
    tl = list(terms)
    arr = (_Term * max(1, len(tl)))(*[_Term(float(c), int(x), int(z)) for c, x, z in tl])
    g = np.zeros(max(1, nparams))
    ev = c_double()
    rc = load().qko_adjoint_grad(_dptr(s), n, circuit.gates, circuit.ngates, p.ctypes.data_as(POINTER(c_int)),
                                 nparams, ctypes.cast(arr, ctypes.c_void_p), len(tl), ctypes.byref(ev), _dptr(g))
    if rc:
        raise RuntimeError("oracle adjoint: unsupported gate")
    return ev.value, g[:nparams]
