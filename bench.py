#!/usr/bin/env python
"""Benchmark of the GPU runner on the 30-qubit random circuit.

Workload (one step): a 30-qubit, 20-layer random circuit -- per layer a
U3(theta, phi, lambda) on every qubit (written as U1 with its 2x2 matrix) then
CZ (CP pi) on brick-pattern neighbour pairs -- applied to |0...0> in
complex128 (a 16 GiB state, larger than L2), through the per-gate path.
Metric: algorithmic HBM GB/s of the circuit (bytes each gate must read and
write, divided by the device time of the step); ms_per_step is the circuit
time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (launched under torch.distributed.run) every rank runs its own
replica of the circuit on its own GPU: the path has no exchange step, so
there is no collective on the data path ("replicas only").
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_QUBITS = 30
N_LAYERS = 20
SEED = 2030
METRIC = "random30_c128_circuit_hbm_gbs"
UNIT = "GB/s"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--qubits", type=int, default=N_QUBITS)
    ap.add_argument("--layers", type=int, default=N_LAYERS)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-fused", action="store_true")
    ap.add_argument("--no-extra", action="store_true", help="skip the other named workloads (QFT-20, HEA-26, 33q c64)")
    return ap.parse_args()


def config_dict(args, world):
    n = args.qubits
    return {"workload": f"random circuit, {n} qubits, {args.layers} layers (U3 on every qubit + brick CZ), "
                        "complex128, per-gate path",
            "qubits": n, "layers": args.layers, "seed": SEED, "state_bytes": 16 << n,
            "l2": "inputs larger than L2 (state >> 126 MB)", "parallelism": f"replicas x{world}",
            "reference_sample": f"the reference arm and cpu_baseline time layer 1 ({n + n // 2} gates) of the "
                                "circuit per step and report its GB/s; every layer has the same gate mix, so the "
                                "rate stands for the whole circuit"}


# ---------------------------------------------------------------------------
# CPU baseline: the unmodified reference MEM runner on the host cores
# ---------------------------------------------------------------------------
def mem_available_bytes():
    try:
        for line in open("/proc/meminfo"):
            if line.startswith("MemAvailable:"):
                return int(line.split()[1]) * 1024
    except OSError:
        pass
    return 0


def cpu_sample(circ, n_gates):
    from subquokka_dev_b200.engine import Circuit
    return Circuit(circ.gate_list()[:n_gates])


def compare_with_file(sv, path):
    """(max |delta amp|, 1 - fidelity) of a device state against a raw
    complex128 state file, streamed through the GPU 1 GiB at a time."""
    import numpy as np
    import oracle
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
        del r, g
    if not np.isfinite(dmax):
        dmax = float("inf")
    return dmax, max(0.0, 1.0 - abs(ov) ** 2 / (nx * ny))


def run_cpu_baseline(circ, n, n_gates, check_gpu=False):
    """Time the reference (oracle/_ref) or, if it was not built, the oracle's C
    port, on the first n_gates gates of the workload.  With check_gpu the
    reference's final state of that sample (the full 2^n amplitudes) is also
    compared with the GPU per-gate path's state for the same gates.  Returns a
    dict."""
    import tempfile
    import numpy as np
    import oracle
    from subquokka_dev_b200.circuits import algorithmic_bytes
    sample = cpu_sample(circ, n_gates)
    sbytes = algorithmic_bytes(sample, n)
    cores = os.cpu_count() or 1
    file_qbit = max(0, int(math.floor(math.log2(cores))))
    threads = 1 << file_qbit
    need = (16 << n) + (2 << 30)
    if mem_available_bytes() < need:
        return {"value": None, "unit": UNIT, "cores": cores, "kind": "reference",
                "sample": f"skipped: host has less than {need >> 30} GiB available"}
    desc = f"first {n_gates} gates (layer 1) of the {n}-qubit circuit, runner span only"
    parity = None
    if oracle.have_reference():
        with tempfile.TemporaryDirectory() as d:
            out = os.path.join(d, "ref_state.bin") if check_gpu else None
            _, secs = oracle.run_reference(n, sample.to_text(), 0, init=None, chunk_qbit=12,
                                           file_qbit=file_qbit, out_path=out)
            if check_gpu:
                from subquokka_dev_b200 import StateVector
                with StateVector(n, "c128") as sv:
                    sv.apply(sample)
                    sv.synchronize()
                    dmax, infid = compare_with_file(sv, out)
                parity = {"gates": n_gates, "qubits": n, "max_abs_damp_gpu_vs_reference": dmax,
                          "one_minus_fidelity": infid, "path": "per-gate complex128 (qk_apply_gates)"}
        kind = "reference"
    else:
        s = np.zeros(1 << n, np.complex128)
        s[0] = 1
        t0 = time.perf_counter()
        oracle.apply_circuit(s, n, sample)
        secs = time.perf_counter() - t0
        kind, threads = "port", cores
    out = {"value": sbytes / secs / 1e9, "unit": UNIT, "cores": threads, "host_cores": cores, "kind": kind,
           "sample": desc, "seconds": secs}
    if parity is not None:
        out["sample_parity"] = parity
    return out


def reference_arm(args, rank, world):
    if rank != 0:
        return 0
    from subquokka_dev_b200 import circuits
    circ = circuits.random_u3_cz(args.qubits, args.layers, SEED)
    n_sample = args.qubits + args.qubits // 2   # the first layer
    for _ in range(args.warmup):
        run_cpu_baseline(circ, args.qubits, 1)
    vals, secs = [], []
    cb = None
    for _ in range(args.steps):
        cb = run_cpu_baseline(circ, args.qubits, n_sample)
        if cb["value"] is None:
            print(json.dumps({"impl": "reference", "unavailable": cb["sample"]}))
            return 0
        vals.append(cb["value"])
        secs.append(cb["seconds"])
    v = statistics.median(vals)
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * statistics.median(secs), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
            "impl": "reference", "config": config_dict(args, world),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cb["cores"], "host_cores": cb["host_cores"],
                             "kind": cb["kind"], "sample": cb["sample"]},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id):
        self.proc = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-i", gpu_id,
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        out, _ = self.proc.communicate(timeout=10)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.splitlines():
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax.append(float(p[2]))
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "samples": len(sm), "reasons": sorted(reasons)}


def load_traffic():
    """dram bytes per launch of the dominant kernel from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "roofline_traffic.json")
    try:
        return json.load(open(p))
    except (OSError, ValueError):
        return {}


def measured_peak_hbm():
    try:
        return float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]), "measured"
    except (OSError, ValueError, KeyError):
        return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def kernel_class(g):
    """Name of the kernel a gate launches (see csrc/qk_engine.cu launch_op)."""
    if g.kind == 9:
        return "k_dense1_lane" if g.q[0] < 5 else "k_dense1_pair"
    if g.kind == 12:
        return "k_phase2"
    return f"kind{g.kind}"


def max_over_ranks(value: float, world: int, device="cuda") -> float:
    """The max of a per-rank number over all ranks (the slowest replica)."""
    if world <= 1:
        return float(value)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(world: int, bytes_per_step: int, steps: int, max_ms: float) -> float:
    """Whole-job GB/s: every rank runs its own replica, timed by the slowest."""
    return world * bytes_per_step * steps / (max_ms / 1e3) / 1e9


def time_device(fn, warmup, steps):
    """Device time (ms) per call of fn, CUDA events on the current stream."""
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def compare_states(a, b):
    """(max |delta amp|, 1 - fidelity) of two device states, on the GPU."""
    import torch
    x, y = a.as_torch(), b.as_torch()
    chunk = 1 << 26
    dmax, ov, nx, ny = 0.0, 0j, 0.0, 0.0
    for i in range(0, x.numel(), chunk):
        xs = x[i:i + chunk].to(torch.complex128)
        ys = y[i:i + chunk].to(torch.complex128)
        dmax = max(dmax, float((xs - ys).abs().max()))
        ov += complex(torch.vdot(xs, ys))
        nx += float(torch.vdot(xs, xs).real)
        ny += float(torch.vdot(ys, ys).real)
    # 1 - F below the rounding of the sums (|values| ~1e-16) reads as 0
    return dmax, max(0.0, 1.0 - abs(ov) ** 2 / (nx * ny))


def fused_variants(args, circ, exact, plain_ms, alg):
    """The same circuit through fused passes, complex128 and complex64, and as
    a subcircuit file (chunk_groups, 12-qubit chunks) through the subcircuit
    path; each is compared with the exact per-gate complex128 state left in
    `exact`."""
    import torch
    from subquokka_dev_b200 import Plan, StateVector
    out = {}
    n = args.qubits
    from subquokka_dev_b200 import chunk_groups
    sub = chunk_groups(circ, n, 12)   # the circuit as a subcircuit file, 12-qubit chunks
    for key, dtype, fw in (("c128", "c128", 0), ("c128_tensor_core", "c128", 6), ("c64", "c64", 0),
                           ("c64_tensor_core", "c64", 6),
                           ("c64_tensor_core_width5", "c64", 5), ("c128_subcircuit_file", "c128", -1),
                           ("c64_subcircuit_file", "c64", -1), ("c64_tensor_core_subcircuit_file", "c64", -6)):
        plan = (Plan(sub, n, dtype, groups=True, fuse_width=-fw if fw < -1 else 0) if fw < 0
                else Plan(circ, n, dtype, fuse_width=fw))
        passes, ops, remaps = plan.stats()
        sv = StateVector(n, dtype)
        sv.set_stream(torch.cuda.current_stream().cuda_stream)

        def run():
            sv.reset()
            plan.apply(sv)
        ms = time_device(run, 2, max(1, args.steps))
        dmax, infid = compare_states(sv, exact)
        amp = 16 if dtype == "c128" else 8
        out[key] = {"ms_per_circuit": ms, "speedup_vs_plain_c128": plain_ms / ms, "passes": passes,
                      "program_ops": ops, "remaps": remaps,
                      "hbm_gbs_passes": passes * 2 * (amp << n) / (ms / 1e3) / 1e9,
                      "max_abs_damp_vs_c128": dmax, "one_minus_fidelity_vs_c128": infid}
        sv.close()
        plan.close()
    return out


def extra_workloads(args):
    """The other named workloads, each timed with CUDA events after warm-up:
    QFT-20 on a seeded random state; QFT-30 as a subcircuit file through the
    subcircuit path against its flat fused plan; the 26-qubit hardware-efficient ansatz
    (12 layers, 624 parameters, ZZ + X Hamiltonian): <H> + adjoint gradient;
    the 33-qubit 24-layer random circuit in complex64 (fused passes), its error
    measured against complex128 on the same circuit family at 28 qubits."""
    import numpy as np
    import torch
    from subquokka_dev_b200 import (Circuit, Plan, StateVector, adjoint_grad, chunk_groups, circuits, make_gate,
                                    zz_x_hamiltonian)
    from subquokka_dev_b200.torch_shim import hea_template
    out = {}
    stream = torch.cuda.current_stream().cuda_stream

    # QFT-20 (L2-resident 16 MiB state)
    n = 20
    init = circuits.random_state(n, 20)
    qft = circuits.qft(n)
    sv = StateVector(n)
    sv.set_stream(stream)
    plan = Plan(qft, n)

    sv.upload(init)
    ms_pg = time_device(lambda: sv.apply(qft), 3, 20)
    graph = sv.capture(qft)   # the same per-gate kernels, one graph launch
    ms_gr = time_device(graph.launch, 3, 20)
    graph.close()
    ms_fu = time_device(lambda: plan.apply(sv), 3, 20)
    out["qft20_c128"] = {"gates": qft.ngates, "per_gate_ms": ms_pg, "per_gate_graph_ms": ms_gr, "fused_ms": ms_fu,
                         "passes": plan.stats()[0], "gates_per_s_per_gate_path": qft.ngates / (ms_pg / 1e3),
                         "gates_per_s_per_gate_graph": qft.ngates / (ms_gr / 1e3)}
    sv.close()
    plan.close()

    # QFT-30 as a subcircuit file (12-qubit chunks, VSWAP groups between the
    # compute groups, written by chunk_groups) through the subcircuit path,
    # against the flat circuit's fused plan
    n = 30
    qft = circuits.qft(n)
    sub = chunk_groups(qft, n, 12)
    nv = sum(1 for i in range(sub.ngates) if sub.gates[i].kind == 14)
    res = {"gates": qft.ngates, "chunk_qbit": 12, "groups": sub.ngroups, "vswaps_in_file": nv}
    states = {}
    for dtype in ("c128", "c64"):
        sv = StateVector(n, dtype)
        sv.set_stream(stream)
        for key, plan in (("subcircuit_file", Plan(sub, n, dtype, groups=True)), ("flat_plan", Plan(qft, n, dtype))):
            def run():
                sv.reset()
                plan.apply(sv)
            ms = time_device(run, 2, max(1, min(args.steps, 5)))
            res[f"{dtype}_{key}_ms"] = ms
            res[f"{dtype}_{key}_passes"] = plan.stats()[0]
            plan.close()
            if dtype == "c128":
                states[key] = sv.download()
        sv.close()
    res["max_abs_diff_file_vs_flat_c128"] = float(np.abs(states["subcircuit_file"] - states["flat_plan"]).max())
    del states
    out["qft30_subcircuit_file"] = res

    # HEA-26 adjoint gradients
    n, layers = 26, 12
    pc = hea_template(n, layers)
    rng = np.random.default_rng(26)
    params = rng.uniform(-np.pi, np.pi, pc.nparams)
    terms = zz_x_hamiltonian(n, rng.standard_normal(n - 1), rng.standard_normal(n))
    circ, idx = pc.bind(params)
    res = {"qubits": n, "layers": layers, "params": pc.nparams, "gates": circ.ngates}
    grads = {}
    peak, _ = measured_peak_hbm()
    from subquokka_dev_b200 import last_sweep
    for dtype, fused in (("c128", False), ("c128", True), ("c64", True)):
        sv = StateVector(n, dtype)
        sv.set_stream(stream)
        box = {"dev": []}

        def run():
            sv.reset()
            box["r"] = adjoint_grad(sv, circ, idx, pc.nparams, terms, -1, fused)
            box["dev"].append(last_sweep(sv))
        ms = time_device(run, 2, 3)
        ev, g, drift = box["r"]
        grads[(dtype, fused)] = g
        key = f"{dtype}_{'fused' if fused else 'per_gate'}"
        # device span of the sweep itself (CUDA events inside the call, host
        # planning excluded), median of the timed calls
        dev = box["dev"][2:]
        dms = statistics.median(d["device_ms"] for d in dev)
        res[key] = {"ms": ms, "grads_per_s": pc.nparams / (ms / 1e3), "device_ms": dms,
                    "grads_per_s_device": pc.nparams / (dms / 1e3), "expval": ev, "drift": drift,
                    "forward_passes": dev[-1]["forward_passes"], "backward_passes": dev[-1]["backward_passes"]}
        if dev[-1]["alg_bytes"] > 0:
            gbs = dev[-1]["alg_bytes"] / (dms / 1e3) / 1e9
            res[key].update({"alg_bytes": dev[-1]["alg_bytes"], "hbm_gbs": gbs, "hbm_frac": gbs / peak})
        sv.close()
    ref = grads[("c128", False)]
    for k, g in grads.items():
        key = f"{k[0]}_{'fused' if k[1] else 'per_gate'}"
        res[key]["max_rel_grad_err_vs_c128_per_gate"] = float(np.abs(g - ref).max() / np.abs(ref).max())
    if not args.no_cpu_baseline:
        # the reference has no gradient code: this project's FP64 CPU adjoint
        # restatement (OpenMP, all host cores) on the first layer of the same ansatz
        import oracle
        pc1 = hea_template(n, 1)
        c1, i1 = pc1.bind(params[:pc1.nparams])
        z = np.zeros(1 << n, np.complex128)
        z[0] = 1
        t0 = time.perf_counter()
        oracle.adjoint_grad(z, n, c1, i1, pc1.nparams, terms)
        secs = time.perf_counter() - t0
        res["cpu_baseline"] = {"grads_per_s": pc1.nparams / secs, "cores": os.cpu_count(), "kind": "port",
                               "sample": f"first layer ({pc1.nparams} parameters) of the 26-qubit ansatz, FP64 C "
                                         "adjoint restatement (the reference computes no gradients)",
                               "seconds": secs}
    out["hea26_adjoint"] = res

    # 33-qubit c64: width-6 dense blocks on the tensor cores (and the CUDA-core
    # register passes for comparison); error at 28 qubits against complex128
    n33, l33 = 33, 24
    c33 = circuits.random_u3_cz(n33, l33, 33)
    res33 = {"qubits": n33, "layers": l33, "gates": c33.ngates, "state_bytes": 8 << n33}
    sv = StateVector(n33, "c64")
    sv.set_stream(stream)
    for key, fw in (("tensor_core_width6", 6), ("cuda_core_passes", 0)):
        p33 = Plan(c33, n33, "c64", fuse_width=fw)

        def run33():
            sv.reset()
            p33.apply(sv)
        ms33 = time_device(run33, 1, 2)
        np33 = p33.stats()[0]
        res33[key] = {"ms_per_circuit": ms33, "passes": np33,
                      "hbm_gbs_passes": np33 * 2 * (8 << n33) / (ms33 / 1e3) / 1e9}
        p33.close()
    sv.close()
    c28 = circuits.random_u3_cz(28, l33, 33)
    a = StateVector(28, "c128")
    a.apply(c28)
    for key, fw in (("tensor_core_width6", 6), ("cuda_core_passes", 0)):
        b = StateVector(28, "c64")
        p28 = Plan(c28, 28, "c64", fuse_width=fw)
        p28.apply(b)
        dmax, infid = compare_states(b, a)
        res33[key].update({"check_qubits": 28, "max_abs_damp_vs_c128": dmax, "one_minus_fidelity_vs_c128": infid})
        b.close()
        p28.close()
    a.close()
    out["random33_c64"] = res33

    # single 6-qubit blocks on a 28-qubit c64 state (2 GiB): one tensor-core
    # pass each, for qubit sets that own qubit 0 (state as the N operand) or not
    n28 = 28
    sv = StateVector(n28, "c64")
    sv.set_stream(stream)
    rng = np.random.default_rng(28)
    lay = {}
    for qs in ((10, 11, 12, 13, 14, 15), (3, 4, 7, 8, 9, 10), (1, 2, 7, 8, 9, 10), (0, 1, 2, 3, 4, 5),
               (0, 1, 21, 22, 26, 27)):
        gates = [make_gate("U1", [q], coeff=circuits.u3_matrix(*rng.uniform(0, 2 * np.pi, 3))) for q in qs]
        gates += [make_gate("CP", [qs[k], qs[k + 1]], np.pi) for k in range(5)]
        pb = Plan(Circuit(gates), n28, "c64", fuse_width=6)
        if pb.stats()[0] != 1:
            raise RuntimeError("expected one dense block")
        ms = time_device(lambda: pb.apply(sv), 3, 10)
        lay[",".join(map(str, qs))] = {"layout": "state_n" if 0 in qs else "state_m", "ms_per_pass": ms,
                                       "hbm_gbs": 2 * (8 << n28) / (ms / 1e3) / 1e9}
        pb.close()
    sv.close()
    out["tensor_core_blocks_28q"] = lay

    # host-resident state: the 32-qubit random circuit (20 layers) with the
    # state in pinned host memory (64 GiB c128) and 2^29-amplitude chunks on
    # the GPU (3 x 8 GiB); checked against the same circuit's fused plan in HBM
    out["host_state_32q_c128"] = host_state_workload(32, 29)

    # batch of 256 variational circuits (14-22 qubits, 4-16 layers), complex64,
    # forward + <H> + adjoint gradients from one CUDA graph; tile shapes autotuned
    from subquokka_dev_b200 import Batch
    items = circuits.variational_batch(256, 2025)
    t0 = time.perf_counter()
    batch = Batch(items, "c64", autotune=True)
    setup_s = time.perf_counter() - t0
    batch.run()
    torch.cuda.synchronize()
    reps = 5
    t1 = time.perf_counter()
    dev_ms = []
    for _ in range(reps):
        ev, grads, drift = batch.run()
        dev_ms.append(batch.timing()[0])   # CUDA events around the graph launch
    wall_ms = (time.perf_counter() - t1) / reps * 1e3
    bms = statistics.median(dev_ms)
    balg = batch.timing()[1]
    # spot check against the single-circuit complex128 path
    from subquokka_dev_b200 import adjoint_grad as _adj
    errs = []
    for c in (0, 128, 255):
        pc, params, terms = items[c]
        circ, idx = pc.bind(params)
        with StateVector(pc.n, "c128") as sv:
            _, g, _ = _adj(sv, circ, idx, pc.nparams, terms, 0, True)
        errs.append(float(np.abs(grads[c] - g).max() / np.abs(g).max()))
    st = batch.stats()
    nparams = sum(pc.nparams for pc, _, _ in items)
    peak, _ = measured_peak_hbm()
    out["batch256_c64"] = {"circuits": 256, "params": nparams, "ms_per_batch": wall_ms,
                           "circuits_per_s": 256 / (wall_ms / 1e3), "grads_per_s": nparams / (wall_ms / 1e3),
                           "device_ms_per_batch": bms, "circuits_per_s_device": 256 / (bms / 1e3),
                           "grads_per_s_device": nparams / (bms / 1e3), "alg_bytes_per_batch": balg,
                           "hbm_gbs": balg / (bms / 1e3) / 1e9, "hbm_frac": balg / (bms / 1e3) / 1e9 / peak,
                           "graph_steps": st["steps"], "launches_per_batch": st["launches"],
                           "tile_shape": [st["tile_bits"], st["reg_bits"], st["adj_tile_bits"], st["adj_reg_bits"]],
                           "setup_s_with_autotune": setup_s, "max_drift": float(drift.max()),
                           "max_rel_grad_err_vs_c128_spot": max(errs)}
    batch.close()
    return out


def sharded_batch(world):
    """The 256-circuit batch (complex64, forward + adjoint) split over all
    ranks by cost (subquokka_dev_b200.sharding): each rank runs one CUDA graph
    over its circuits, one all-reduce gathers every result on every rank.
    circuits/s = 256 / the slowest rank's device time (strong scaling: the
    batch is fixed, the ranks share it)."""
    import torch
    from subquokka_dev_b200 import circuits
    from subquokka_dev_b200.sharding import ShardedBatch
    items = circuits.variational_batch(256, 2025)
    sb = ShardedBatch(items, "c64", device=torch.device("cuda", torch.cuda.current_device()))
    for _ in range(2):
        sb.run()
    ms = []
    for _ in range(5):
        sb.run()
        ms.append(sb.device_ms())
    local = statistics.median(ms)
    worst = max_over_ranks(local, world)
    nparams = sum(pc.nparams for pc, _, _ in items)
    out = {"circuits": 256, "ranks": world, "scaling": "strong", "circuits_on_rank0": len(sb.mine),
           "max_rank_device_ms": worst, "circuits_per_s": 256 / (worst / 1e3), "grads_per_s": nparams / (worst / 1e3),
           "collective": "one all_reduce of the results per run (no data-path exchange)"}
    sb.close()
    return out


def host_state_workload(n, L):
    """qk_hsv_*: a state in pinned host memory, the gates on the GPU chunk by
    chunk; device time (CUDA events, first copy-in to last copy-out), the
    bytes moved over the host link, and the in-HBM fused plan of the same
    circuit for comparison (max |delta amp| between the two)."""
    import numpy as np
    import torch
    from subquokka_dev_b200 import HostStateVector, Plan, StateVector, circuits
    need = (16 << n) + (24 << 30)
    if mem_available_bytes() < need:
        return {"skipped": f"host has less than {need >> 30} GiB available"}
    circ = circuits.random_u3_cz(n, 20, SEED)
    t0 = time.perf_counter()
    hs = HostStateVector(n, L, "c128")
    setup_s = time.perf_counter() - t0
    hs.apply(circ)
    st = hs.stats()
    res = {"qubits": n, "chunk_qubits": L, "gates": circ.ngates, "state_bytes": 16 << n, "segments": st["segments"],
           "device_ms": st["device_ms"], "link_bytes": st["link_bytes"],
           "link_gbs_both_directions": st["link_bytes"] / (st["device_ms"] / 1e3) / 1e9,
           "setup_s_pinned_alloc": setup_s}
    sv = StateVector(n, "c128")
    sv.set_stream(torch.cuda.current_stream().cuda_stream)
    plan = Plan(circ, n, "c128")

    def run():
        sv.reset()
        plan.apply(sv)
    res["in_hbm_fused_ms"] = time_device(run, 1, 1)
    host = hs.view()
    x = sv.as_torch()
    piece = 1 << 26
    dmax = 0.0
    for i in range(0, x.numel(), piece):
        h = torch.from_numpy(host[i:i + piece]).to(x.device)
        dmax = max(dmax, float((h - x[i:i + piece]).abs().max()))
        del h
    res["max_abs_damp_vs_in_hbm"] = dmax
    plan.close()
    sv.close()
    hs.close()
    return res


def sharded_state(world, layers):
    """One state over all ranks (ShardedStateVector): the random circuit on
    30 + log2(N) qubits, 2^30 complex128 amplitudes a rank (weak scaling),
    exchanges by NCCL all-to-all; the slowest rank's device time."""
    import torch
    import torch.distributed as dist
    from subquokka_dev_b200 import circuits
    from subquokka_dev_b200.sharding import ShardedStateVector
    g = world.bit_length() - 1
    if world & (world - 1):
        return {"skipped": "the number of ranks is not a power of two"}
    n = 30 + g
    circ = circuits.random_u3_cz(n, layers, SEED)
    sv = ShardedStateVector(n, "c128")
    dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    sv.apply(circ)
    e1.record()
    torch.cuda.synchronize()
    worst = max_over_ranks(e0.elapsed_time(e1), world)
    out = {"qubits": n, "ranks": world, "scaling": "weak", "amplitudes_per_rank": 1 << 30, "gates": circ.ngates,
           "exchanges": sv.exchanges, "max_rank_ms": worst, "gates_per_s": circ.ngates / (worst / 1e3),
           "timed": "one apply: host planning of each segment, fused passes, all-to-all exchanges"}
    sv.close()
    return out


def our_arm(args, rank, world):
    import numpy as np
    import torch
    import torch.distributed as dist
    from subquokka_dev_b200 import StateVector, _lib, circuits
    from subquokka_dev_b200._lib import check

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    n = args.qubits
    circ = circuits.random_u3_cz(n, args.layers, SEED)
    alg = circuits.algorithmic_bytes(circ, n)
    S = 16 << n
    lib = _lib.load()
    sv = StateVector(n, "c128")
    sv.set_stream(torch.cuda.current_stream().cuda_stream)
    gate_ms = (ctypes.c_float * circ.ngates)()

    def step(timed=False):
        sv.reset()
        if timed:
            check(lib.qk_apply_gates_timed(sv.h, circ.gates, circ.ngates, gate_ms))
        else:
            sv.apply(circ)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        uuid = str(dev)
    sampler = ClockSampler(uuid)
    time.sleep(0.5)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    per_kernel = {}
    ev0.record()
    for _ in range(args.steps):
        step(timed=True)
        for i, g in enumerate(circ.gate_list()):
            per_kernel.setdefault(kernel_class(g), []).append(gate_ms[i])
    ev1.record()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = sampler.stop()
    total_ms = max_over_ranks(ev0.elapsed_time(ev1), world)
    ms_per_step = total_ms / args.steps
    value = replica_throughput(world, alg, args.steps, total_ms)

    # dominant kernel: the dense one-qubit sweep on a high qubit (U1, 2S bytes)
    peak, peak_kind = measured_peak_hbm()
    shares = {k: sum(v) for k, v in per_kernel.items()}
    tot = sum(shares.values())
    dom = "k_dense1_pair"
    dom_ms = statistics.mean(per_kernel[dom])
    achieved = 2 * S / (dom_ms / 1e3) / 1e9
    traffic = load_traffic().get(dom)
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": f"{peak_kind} hbm_gbs (copy)",
                "traffic": traffic, "algorithmic_bytes_per_launch": 2 * S,
                "avg_launch_ms": dom_ms,
                "kernel_share": {k: v / tot for k, v in sorted(shares.items())},
                "kernel_gbs": {k: (2 * S if k.startswith("k_dense1") else S // 2) / (statistics.mean(v) / 1e3) / 1e9
                               for k, v in per_kernel.items()}}
    launches = args.steps * (circ.ngates + 1)
    # the fused forms and the other workloads are single-GPU measurements:
    # a run on N > 1 GPUs (replicas of the timed step) skips them and runs
    # the two multi-GPU legs instead, so that it holds the GPUs briefly
    variants = {} if (args.no_fused or world > 1) else fused_variants(args, circ, sv, ms_per_step, alg)
    extra = {} if (args.no_extra or rank != 0 or world > 1) else None
    sharded = sharded_st = None
    if world > 1 and not args.no_extra:
        # every rank takes part; an error raised on every rank alike is
        # recorded instead of ending the run
        try:
            sharded = sharded_batch(world)
        except Exception as exc:
            sharded = {"error": f"{type(exc).__name__}: {exc}"[:300]}
        try:
            sharded_st = sharded_state(world, args.layers)
        except Exception as exc:
            sharded_st = {"error": f"{type(exc).__name__}: {exc}"[:300]}

    # end to end through the public API: host gate records in, final state out to pinned host memory
    e2e = None
    if not args.no_e2e:
        try:
            host = torch.empty(2 << n, dtype=torch.float64, pin_memory=True)
            pinned = True
        except Exception:
            host = torch.empty(2 << n, dtype=torch.float64)
            pinned = False
        hp = ctypes.cast(host.data_ptr(), ctypes.POINTER(ctypes.c_double))
        e2e_steps = max(1, min(args.steps, 2))
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            sv.reset()
            sv.apply(circ)
            check(lib.qk_sv_download(sv.h, hp))
        el = max_over_ranks(time.perf_counter() - t0, world)
        import ctypes as _ct
        e2e = {"value": world * alg * e2e_steps / el / 1e9, "unit": UNIT,
               "h2d_bytes_per_step": _ct.sizeof(circ.gates._type_) * circ.ngates,
               "d2h_bytes_per_step": S, "ms_per_step": 1e3 * el / e2e_steps,
               "host_buffer": "pinned" if pinned else "pageable"}
        del host
    sv.close()
    if extra is None:
        extra = extra_workloads(args)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = run_cpu_baseline(circ, n, n + n // 2, check_gpu=True)
        cpu.pop("seconds", None)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
                "config": config_dict(args, world), "circuit_seconds": ms_per_step / 1e3,
                "gates_per_s": world * circ.ngates / (ms_per_step / 1e3),
                "hbm_frac_of_peak": value / peak,
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks,
                "gpu_launches": launches, "fused": variants, "workloads": extra}
        if sharded is not None:
            line["batch256_sharded"] = sharded
        if sharded_st is not None:
            line["random_sharded_state"] = sharded_st
        # last, so that a reader of the line's tail sees every target at once
        line["summary"] = summarize(line, peak)
        print(json.dumps(line))
    return 0


def summarize(line, peak):
    """Compact view of the figures the targets are set on: the plain
    complex128 path against HBM roofline, the fused forms' speed-up and error,
    the adjoint and batch rates with their HBM fractions."""
    r = lambda x, k=4: None if x is None else float(f"{x:.{k}g}")
    out = {"plain_c128_s": r(line["circuit_seconds"]), "plain_c128_hbm_frac": r(line["hbm_frac_of_peak"], 3),
           "plain_c128_kernel_frac": r(line["roofline"]["frac"], 3)}
    f = line.get("fused") or {}
    for key, name in (("c64_tensor_core", "fused_c64_tc"), ("c128_tensor_core", "fused_c128_tc"),
                      ("c128", "fused_c128"), ("c64", "fused_c64")):
        if key in f:
            v = f[key]
            out[name] = {"s": r(v["ms_per_circuit"] / 1e3), "x_vs_plain": r(v["speedup_vs_plain_c128"], 3),
                         "one_minus_F": r(v["one_minus_fidelity_vs_c128"], 2),
                         "max_damp": r(v["max_abs_damp_vs_c128"], 2), "hbm_frac": r(v["hbm_gbs_passes"] / peak, 3)}
    w = line.get("workloads") or {}
    h = w.get("hea26_adjoint")
    if h:
        out["hea26_adjoint"] = {k: {"grads_per_s": r(h[k]["grads_per_s"]), "device_ms": r(h[k]["device_ms"]),
                                    "hbm_frac": r(h[k].get("hbm_frac"), 3),
                                    "rel_err_vs_c128": r(h[k]["max_rel_grad_err_vs_c128_per_gate"], 2)}
                                for k in ("c128_fused", "c64_fused") if k in h}
    b = w.get("batch256_c64")
    if b:
        out["batch256_c64"] = {"circuits_per_s": r(b["circuits_per_s"]), "grads_per_s": r(b["grads_per_s"]),
                               "device_ms": r(b["device_ms_per_batch"]), "hbm_frac": r(b["hbm_frac"], 3)}
    q = w.get("random33_c64", {}).get("tensor_core_width6")
    if q:
        out["random33_c64_tc"] = {"s": r(q["ms_per_circuit"] / 1e3), "hbm_frac": r(q["hbm_gbs_passes"] / peak, 3),
                                  "one_minus_F_28q": r(q["one_minus_fidelity_vs_c128"], 2)}
    hs = w.get("host_state_32q_c128")
    if hs and "segments" in hs:
        out["host_state_32q_c128"] = {"s": r(hs["device_ms"] / 1e3), "segments": hs["segments"],
                                      "link_gbs": r(hs["link_gbs_both_directions"]),
                                      "in_hbm_s": r(hs["in_hbm_fused_ms"] / 1e3),
                                      "max_damp_vs_in_hbm": r(hs["max_abs_damp_vs_in_hbm"], 2)}
    cb = line.get("cpu_baseline") or {}
    if cb.get("value"):
        out["cpu_reference_gbs"] = r(cb["value"])
        out["cpu_threads"] = cb.get("cores")
        sp = cb.get("sample_parity")
        if sp:
            out["parity_sample_max_damp_vs_reference"] = sp["max_abs_damp_gpu_vs_reference"]
    return out


def main():
    args = parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        # the reference is CPU code: rank 0 alone times it, other ranks exit
        return reference_arm(args, rank, world)
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        return our_arm(args, rank, world)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
