"""Host-side mirror of the reference's runner interface over the C ABI.

``Simulator(ini, cir).run()`` mirrors the reference's ``Simulator`` class
(src/simulator.hpp:51-83, src/simulator.cpp:671-724): it reads the same .ini
and circuit.txt files, runs the circuit on the GPU runner and reports the
runner-only time.  ``StateVector`` is the device-resident state that replaces
``MEM_Runner::buffer`` (src/MEM_Runner.hpp:27).  Every call goes through
libquokka_gpu.so; nothing here computes amplitudes on the CPU.
"""
from __future__ import annotations

import ctypes
from ctypes import POINTER, byref, c_double, c_int, c_int32, c_size_t, c_void_p
from typing import Iterable, Sequence

import numpy as np

from . import _lib
from ._lib import GATE_KINDS, KIND_NAMES, QK_C64, QK_C128, QkConfig, QkGate, check

DTYPES = {"c128": QK_C128, "c64": QK_C64, QK_C128: QK_C128, QK_C64: QK_C64}


# ---------------------------------------------------------------------------
# gates and circuits
# ---------------------------------------------------------------------------
def make_gate(name: str, qubits: Sequence[int], param: float = 0.0, coeff=None) -> QkGate:
    """Build one gate record (the struct qk_gate of include/quokka_gpu.h)."""
    g = QkGate()
    g.kind = GATE_KINDS[name]
    g.nq = len(qubits)
    for i, q in enumerate(qubits):
        g.q[i] = int(q)
    g.param = float(param)
    if coeff is not None:
        flat = []
        for z in np.asarray(coeff, dtype=np.complex128).ravel():
            flat += [float(z.real), float(z.imag)]
        for i, v in enumerate(flat):
            g.coeff[i] = v
    return g


def gate_line(g: QkGate) -> str:
    """circuit.txt line of a gate, with round-trip exact floats."""
    name = KIND_NAMES[g.kind]
    qs = [g.q[i] for i in range(g.nq)]
    if name in ("VSWAP", "MPI_VSWAP"):
        k = g.nq // 2
        name = f"{name}_{k}_{k}"
    parts = [name] + [str(q) for q in qs]
    if name in ("P", "RX", "RY", "RZ", "CP", "RZZ"):
        parts.append(repr(float(g.param)))
    ncoef = {"U1": 4, "U2": 16}.get(name, 0)
    parts += [repr(float(g.coeff[i])) for i in range(2 * ncoef)]
    return " ".join(parts)


class Circuit:
    """A parsed gate list plus group sizes (one group per gate for flat files)."""

    def __init__(self, gates: Iterable[QkGate], group_sizes: Sequence[int] | None = None):
        gl = list(gates)
        self.gates = (QkGate * max(1, len(gl)))(*gl)
        self.ngates = len(gl)
        gs = list(group_sizes) if group_sizes is not None else [1] * len(gl)
        if sum(gs) != len(gl):
            raise ValueError("group sizes do not add up to the gate count")
        self.group_sizes = (c_int32 * max(1, len(gs)))(*gs)
        self.ngroups = len(gs)

    @classmethod
    def _from_handle(cls, h: c_void_p) -> "Circuit":
        lib = _lib.load()
        try:
            ng = lib.qk_circuit_num_gates(h)
            gp = lib.qk_circuit_gates(h)
            gates = [QkGate.from_buffer_copy(gp[i]) for i in range(ng)]
            nG = lib.qk_circuit_num_groups(h)
            sp = lib.qk_circuit_group_sizes(h)
            sizes = [sp[i] for i in range(nG)]
        finally:
            lib.qk_circuit_destroy(h)
        return cls(gates, sizes)

    @classmethod
    def load(cls, path: str, is_subcircuit: int, total_qbit: int) -> "Circuit":
        h = c_void_p()
        check(_lib.load().qk_circuit_load(path.encode(), int(is_subcircuit), int(total_qbit), byref(h)))
        return cls._from_handle(h)

    @classmethod
    def parse(cls, text: str, is_subcircuit: int, total_qbit: int) -> "Circuit":
        h = c_void_p()
        check(_lib.load().qk_circuit_parse(text.encode(), int(is_subcircuit), int(total_qbit), byref(h)))
        return cls._from_handle(h)

    def gate_list(self) -> list[QkGate]:
        return [self.gates[i] for i in range(self.ngates)]

    def to_text(self, is_subcircuit: bool = False) -> str:
        lines = []
        if not is_subcircuit:
            lines = [gate_line(self.gates[i]) for i in range(self.ngates)]
        else:
            k = 0
            for gi in range(self.ngroups):
                n = self.group_sizes[gi]
                lines.append(str(n))
                lines += [gate_line(self.gates[k + j]) for j in range(n)]
                k += n
        return "\n".join(lines) + "\n" if lines else ""


def chunk_groups(circuit: Circuit, n: int, chunk_qbit: int = 12) -> Circuit:
    """The subcircuit file of a flat circuit for the reference's subcircuit
    runner (the output subcircuitFinder makes, subcircuitFinder/finder.cpp:
    771-877): compute groups on bit positions below chunk_qbit, VSWAP_1_1 /
    VSWAP_2_2 groups between them, the state back in the input's layout at
    the end.  ``.to_text(True)`` is the file's text."""
    h = c_void_p()
    check(_lib.load().qk_circuit_chunk_groups(circuit.gates, circuit.ngates, int(n), int(chunk_qbit), byref(h)))
    return Circuit._from_handle(h)


def parse_line(line: str, total_qbit: int) -> QkGate:
    g = QkGate()
    check(_lib.load().qk_gate_parse_line(line.encode(), int(total_qbit), byref(g)))
    return g


def gate_matrix(g: QkGate) -> np.ndarray:
    """Dense FP64 matrix of a gate over its targets (little-endian target order)."""
    dim = 1 << g.nq
    out = (c_double * (2 * dim * dim))()
    d = c_int()
    check(_lib.load().qk_gate_matrix(byref(g), out, byref(d)))
    a = np.frombuffer(out, dtype=np.float64).copy().view(np.complex128)
    return a.reshape(dim, dim)


# ---------------------------------------------------------------------------
# configuration
# ---------------------------------------------------------------------------
class Config:
    """The [system] section of an .ini file (setSEG/setENV keys + engine keys)."""

    def __init__(self, path: str):
        self.raw = QkConfig()
        check(_lib.load().qk_config_load(path.encode(), byref(self.raw)))

    def __getattr__(self, name):
        raw = object.__getattribute__(self, "raw")
        v = getattr(raw, name)
        return v.decode() if isinstance(v, bytes) else v


# ---------------------------------------------------------------------------
# device state
# ---------------------------------------------------------------------------
class StateVector:
    """A 2^n-amplitude state resident in HBM (complex128 or complex64)."""

    def __init__(self, nqubits: int, dtype="c128"):
        self._lib = _lib.load()
        self.h = c_void_p()
        check(self._lib.qk_sv_create(int(nqubits), DTYPES[dtype], byref(self.h)))
        self.nqubits = int(nqubits)
        self.dtype = DTYPES[dtype]

    def close(self) -> None:
        if self.h:
            self._lib.qk_sv_destroy(self.h)
            self.h = c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def namp(self) -> int:
        return 1 << self.nqubits

    def info(self):
        n, dt, p, b = c_int(), c_int(), c_void_p(), c_size_t()
        check(self._lib.qk_sv_info(self.h, byref(n), byref(dt), byref(p), byref(b)))
        return n.value, dt.value, p.value, b.value

    @property
    def device_ptr(self) -> int:
        return self.info()[2]

    @property
    def nbytes(self) -> int:
        return self.info()[3]

    def reset(self) -> None:
        check(self._lib.qk_sv_reset(self.h))

    @property
    def __cuda_array_interface__(self):
        return {"shape": (self.namp,), "typestr": "<c16" if self.dtype == QK_C128 else "<c8",
                "data": (self.device_ptr, False), "version": 3}

    def as_torch(self):
        """Zero-copy torch view of the device state (complex128/complex64)."""
        import torch
        return torch.as_tensor(self, device="cuda")

    def apply_plan(self, plan: "Plan") -> None:
        plan.apply(self)

    def upload(self, state: np.ndarray) -> None:
        a = np.ascontiguousarray(state, dtype=np.complex128)
        if a.size != self.namp:
            raise ValueError(f"state has {a.size} amplitudes, expected {self.namp}")
        check(self._lib.qk_sv_upload(self.h, a.ctypes.data_as(POINTER(c_double))))

    def download(self, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.empty(self.namp, dtype=np.complex128)
        check(self._lib.qk_sv_download(self.h, out.ctypes.data_as(POINTER(c_double))))
        return out

    def save(self, path: str) -> None:
        """Write the state as raw little-endian complex128 (dump_format=bin)."""
        check(self._lib.qk_sv_save(self.h, str(path).encode()))

    def load(self, path: str) -> None:
        """Read a state file written by save() or dump_format=bin."""
        check(self._lib.qk_sv_load(self.h, str(path).encode()))

    def set_stream(self, stream_ptr: int | None) -> None:
        check(self._lib.qk_sv_set_stream(self.h, c_void_p(stream_ptr or 0)))

    def synchronize(self) -> None:
        check(self._lib.qk_sv_synchronize(self.h))

    def release_workspace(self) -> None:
        """Free the device memory adjoint sweeps keep with this state."""
        check(self._lib.qk_sv_release_workspace(self.h))

    def apply(self, circuit: Circuit) -> None:
        """Per-gate path (MEM_Runner::run(vector<Gate*>&))."""
        check(self._lib.qk_apply_gates(self.h, circuit.gates, circuit.ngates))

    def capture(self, circuit: Circuit) -> "GateGraph":
        """The per-gate path for `circuit` captured as a CUDA graph on this
        state: `graph.launch()` applies the circuit again with one launch."""
        return GateGraph(self, circuit)

    def apply_groups(self, circuit: Circuit) -> None:
        """Subcircuit path (MEM_Runner::run(vector<vector<Gate*>>&))."""
        check(self._lib.qk_apply_groups(self.h, circuit.gates, circuit.group_sizes, circuit.ngroups))


class GateGraph:
    """qk_graph_*: the per-gate kernels of a circuit as one CUDA graph bound
    to a state (close it before the state)."""

    def __init__(self, sv: "StateVector", circuit: Circuit):
        self._lib = _lib.load()
        self.sv = sv
        self.h = c_void_p()
        check(self._lib.qk_graph_create(sv.h, circuit.gates, circuit.ngates, byref(self.h)))

    def launch(self) -> None:
        check(self._lib.qk_graph_launch(self.h))

    def close(self) -> None:
        if self.h:
            self._lib.qk_graph_destroy(self.h)
            self.h = c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class Plan:
    """A fused plan: the circuit cut into passes, each one HBM read + write of
    the state (qk_plan_create / qk_plan_create_groups)."""

    def __init__(self, circuit: Circuit, nqubits: int, dtype="c128", tile_bits: int = 0, reg_bits: int = 0,
                 groups: bool = False, fuse_width: int = 0):
        self._lib = _lib.load()
        o = _lib.QkPlanOpts()
        o.dtype = DTYPES[dtype]
        o.tile_bits = int(tile_bits)
        o.reg_bits = int(reg_bits)
        o.fuse_width = int(fuse_width)
        self.h = c_void_p()
        if groups:
            check(self._lib.qk_plan_create_groups(circuit.gates, circuit.group_sizes, circuit.ngroups, int(nqubits),
                                                  byref(o), byref(self.h)))
        else:
            check(self._lib.qk_plan_create(circuit.gates, circuit.ngates, int(nqubits), byref(o), byref(self.h)))
        self.nqubits = int(nqubits)
        self.dtype = DTYPES[dtype]

    def stats(self):
        """(passes, program ops, register re-mappings)."""
        a, b, c = c_size_t(), c_size_t(), c_size_t()
        check(self._lib.qk_plan_stats(self.h, byref(a), byref(b), byref(c)))
        return a.value, b.value, c.value

    def apply(self, sv: "StateVector") -> None:
        check(self._lib.qk_plan_apply(sv.h, self.h))

    def dense_block(self, k: int):
        """(qubits, 64 x 64 unitary or None, is_perm) of block k of a fuse_width = 5 or 6 plan."""
        qs = (c_int32 * 6)()
        u = np.zeros(2 * 64 * 64)
        perm = c_int()
        check(self._lib.qk_plan_dense_block(self.h, int(k), qs, u.ctypes.data_as(POINTER(c_double)), byref(perm)))
        qlist = [q for q in qs if q >= 0]
        return qlist, (None if perm.value else u.view(np.complex128).reshape(64, 64)), bool(perm.value)

    def close(self) -> None:
        if self.h:
            self._lib.qk_plan_destroy(self.h)
            self.h = c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# observables and gradients
# ---------------------------------------------------------------------------
def pauli_terms(terms) -> "ctypes.Array":
    """[(coeff, x_mask, z_mask), ...] -> qk_pauli_term array."""
    tl = list(terms)
    arr = (_lib.QkPauliTerm * max(1, len(tl)))()
    for i, (c, x, z) in enumerate(tl):
        arr[i].coeff = float(c)
        arr[i].x_mask = int(x)
        arr[i].z_mask = int(z)
    arr._n = len(tl)
    return arr


def zz_x_hamiltonian(n: int, J, h):
    """H = sum_i J_i Z_i Z_{i+1} + sum_i h_i X_i as (coeff, x_mask, z_mask) terms."""
    terms = [(float(J[i]), 0, (1 << i) | (1 << (i + 1))) for i in range(n - 1)]
    terms += [(float(h[i]), 1 << i, 0) for i in range(n)]
    return terms


def expval(sv: "StateVector", terms) -> float:
    arr = pauli_terms(terms)
    out = c_double()
    check(_lib.load().qk_expval_pauli(sv.h, arr, arr._n, byref(out)))
    return out.value


def adjoint_grad(sv: "StateVector", circuit: Circuit, param_index, nparams: int, terms, checkpoints: int = -1,
                 fused: bool = False):
    """(<H>, gradient, checkpoint drift) of H after `circuit` applied to sv's
    state; gate i is trainable when param_index[i] >= 0 (RX/RY/RZ).  fused:
    fused forward passes and two-state adjoint passes instead of one kernel
    per gate."""
    pidx = np.ascontiguousarray(param_index, dtype=np.int32)
    if pidx.size != circuit.ngates:
        raise ValueError("param_index needs one entry per gate")
    arr = pauli_terms(terms)
    grad = np.zeros(max(1, nparams), dtype=np.float64)
    ev, drift = c_double(), c_double()
    fn = _lib.load().qk_adjoint_grad_fused if fused else _lib.load().qk_adjoint_grad
    check(fn(sv.h, circuit.gates, circuit.ngates, pidx.ctypes.data_as(POINTER(c_int32)),
                                      int(nparams), arr, arr._n, int(checkpoints), byref(ev),
                                      grad.ctypes.data_as(POINTER(c_double)), byref(drift)))
    return ev.value, grad[:nparams], drift.value


class HostStateVector:
    """A state too large for HBM (qk_hsv_*): 2^n amplitudes in pinned host
    memory, the gates run on the GPU chunk by chunk, 2^chunk_qubits
    amplitudes at a time.  The replacement of the reference's IO runner
    (src/IO_Runner.cpp:309-488)."""

    def __init__(self, nqubits: int, chunk_qubits: int, dtype="c128"):
        self._lib = _lib.load()
        self.h = c_void_p()
        check(self._lib.qk_hsv_create(int(nqubits), int(chunk_qubits), DTYPES[dtype], byref(self.h)))
        self.nqubits, self.chunk_qubits, self.dtype = int(nqubits), int(chunk_qubits), DTYPES[dtype]

    def view(self) -> np.ndarray:
        """Zero-copy numpy view of the host amplitudes (complex128 / complex64)."""
        ct = ctypes.c_double if self.dtype == QK_C128 else ctypes.c_float
        p = ctypes.cast(self._lib.qk_hsv_data(self.h), POINTER(ct))
        a = np.ctypeslib.as_array(p, shape=(2 << self.nqubits,))
        return a.view(np.complex128 if self.dtype == QK_C128 else np.complex64)

    def reset(self) -> None:
        check(self._lib.qk_hsv_reset(self.h))

    def apply(self, circuit: Circuit) -> None:
        check(self._lib.qk_hsv_apply_gates(self.h, circuit.gates, circuit.ngates))

    def stats(self) -> dict:
        sg, ms, nb = c_int(), c_double(), c_double()
        check(self._lib.qk_hsv_stats(self.h, byref(sg), byref(ms), byref(nb)))
        return {"segments": sg.value, "device_ms": ms.value, "link_bytes": nb.value}

    def close(self) -> None:
        if self.h:
            self._lib.qk_hsv_destroy(self.h)
            self.h = c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def ooc_segments(circuit: Circuit, nqubits: int, chunk_qubits: int):
    """The segments qk_hsv_apply_gates would run: [(local qubit mask, [gate
    indices in execution order]), ...] (host only)."""
    lib = _lib.load()
    ns = c_size_t()
    check(lib.qk_ooc_segments(circuit.gates, circuit.ngates, int(nqubits), int(chunk_qubits), None, None, None, 0,
                              byref(ns)))
    k = ns.value
    masks = (ctypes.c_uint64 * max(1, k))()
    sizes = (c_int32 * max(1, k))()
    order = (c_int32 * max(1, circuit.ngates))()
    check(lib.qk_ooc_segments(circuit.gates, circuit.ngates, int(nqubits), int(chunk_qubits), masks, sizes, order,
                              k, byref(ns)))
    out, pos = [], 0
    for i in range(k):
        out.append((int(masks[i]), [int(order[pos + j]) for j in range(sizes[i])]))
        pos += sizes[i]
    return out


def last_sweep(sv: "StateVector") -> dict:
    """Device time (ms, CUDA events), algorithmic bytes (0 = not counted) and
    pass counts of the last adjoint sweep on sv (qk_sv_last_sweep)."""
    ms, nb, f, b = c_double(), c_double(), c_int(), c_int()
    check(_lib.load().qk_sv_last_sweep(sv.h, byref(ms), byref(nb), byref(f), byref(b)))
    return {"device_ms": ms.value, "alg_bytes": nb.value, "forward_passes": f.value, "backward_passes": b.value}


class Batch:
    """Many variational circuits, <H> and adjoint gradients of each, from one
    CUDA graph (qk_batch_*).  items: [(ParamCircuit, params, terms), ...]."""

    def __init__(self, items, dtype="c64", autotune: bool = False, tile_bits: int = 0, reg_bits: int = 0,
                 adj_tile_bits: int = 0, adj_reg_bits: int = 0):
        self._lib = _lib.load()
        nq, gates, gcount, pidx, pcount, terms, tcount = [], [], [], [], [], [], []
        self.param_counts = []
        for pc, params, tl in items:
            circ, idx = pc.bind(np.asarray(params, dtype=np.float64))
            nq.append(pc.n)
            gates += circ.gate_list()
            gcount.append(circ.ngates)
            pidx += list(idx)
            pcount.append(pc.nparams)
            self.param_counts.append(pc.nparams)
            terms += list(tl)
            tcount.append(len(tl))
        self.ncirc = len(items)
        self.nparams = int(sum(pcount))
        self._gates = (QkGate * len(gates))(*gates)
        arr_t = pauli_terms(terms)
        o = _lib.QkBatchOpts()
        o.dtype = DTYPES[dtype]
        o.autotune = int(autotune)
        o.tile_bits, o.reg_bits, o.adj_tile_bits, o.adj_reg_bits = tile_bits, reg_bits, adj_tile_bits, adj_reg_bits
        self.h = c_void_p()
        check(self._lib.qk_batch_create(
            self.ncirc, (c_int32 * self.ncirc)(*nq), self._gates, (c_size_t * self.ncirc)(*gcount),
            (c_int32 * len(pidx))(*pidx), (c_size_t * self.ncirc)(*pcount), arr_t,
            (c_size_t * self.ncirc)(*tcount), byref(o), byref(self.h)))

    def run(self):
        """(expvals[ncirc], [grad of circuit c], drift[ncirc])."""
        ev = np.zeros(self.ncirc)
        g = np.zeros(max(1, self.nparams))
        dr = np.zeros(self.ncirc)
        check(self._lib.qk_batch_run(self.h, ev.ctypes.data_as(POINTER(c_double)), g.ctypes.data_as(POINTER(c_double)),
                                     dr.ctypes.data_as(POINTER(c_double))))
        grads, k = [], 0
        for n in self.param_counts:
            grads.append(g[k:k + n].copy())
            k += n
        return ev, grads, dr

    def set_params(self, params_per_circuit) -> None:
        flat = np.concatenate([np.asarray(p, dtype=np.float64) for p in params_per_circuit])
        check(self._lib.qk_batch_set_params(self.h, flat.ctypes.data_as(POINTER(c_double))))

    def timing(self):
        """(device ms of the last run, algorithmic bytes of one run) (qk_batch_timing)."""
        ms, nb = c_double(), c_double()
        check(self._lib.qk_batch_timing(self.h, byref(ms), byref(nb)))
        return ms.value, nb.value

    def stats(self):
        v = [c_int() for _ in range(6)]
        check(self._lib.qk_batch_stats(self.h, *[byref(x) for x in v]))
        k = ["steps", "launches", "tile_bits", "reg_bits", "adj_tile_bits", "adj_reg_bits"]
        return {a: b.value for a, b in zip(k, v)}

    def close(self) -> None:
        if self.h:
            self._lib.qk_batch_destroy(self.h)
            self.h = c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def apply_gates_dev(ptr: int, nqubits: int, dtype, circuit: Circuit, stream_ptr: int | None = None) -> None:
    """Per-gate path on caller-owned device memory (e.g. a torch tensor)."""
    check(_lib.load().qk_apply_gates_dev(c_void_p(ptr), int(nqubits), DTYPES[dtype], circuit.gates,
                                         circuit.ngates, c_void_p(stream_ptr or 0)))


# ---------------------------------------------------------------------------
# the reference-facing runner
# ---------------------------------------------------------------------------
class Simulator:
    """``Simulator(ini, cir)`` + ``run()`` with runner_type=GPU.

    Mirrors src/simulator.cpp:708-724 (construction: read ini, parse circuit,
    allocate the |0...0> state) and :671-706 (run: time the runner span only).
    """

    def __init__(self, ini: str, cir: str):
        self.config = Config(ini)
        if self.config.runner_type not in ("GPU", "MEM"):
            raise _lib.QkError(-1, f"[Config File]: {self.config.runner_type} runner not found.")
        if self.config.mpi_qbit:
            raise _lib.QkError(-8, "mpi_qbit > 0 is not supported by the GPU runner")
        self.circuit = Circuit.load(cir, self.config.is_subcircuit, self.config.total_qbit)
        self.state = StateVector(self.config.total_qbit, self.config.precision)
        if self.config.init_file:
            self.state.load(self.config.init_file)

    def run(self) -> float:
        sec = c_double()
        h = c_void_p()
        lib = _lib.load()
        # qk_run takes the parsed circuit handle; rebuild one from our records
        text = self.circuit.to_text(bool(self.config.is_subcircuit))
        check(lib.qk_circuit_parse(text.encode(), self.config.is_subcircuit, self.config.total_qbit, byref(h)))
        try:
            check(lib.qk_run(byref(self.config.raw), h, self.state.h, byref(sec)))
        finally:
            lib.qk_circuit_destroy(h)
        return sec.value
