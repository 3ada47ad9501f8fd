"""Helpers for reading the golden fixtures (tests/golden/*.npz)."""
import glob
import os

import numpy as np

GOLDEN_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def names():
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN_DIR, "*.npz")))


def load(name):
    z = np.load(os.path.join(GOLDEN_DIR, name + ".npz"))
    rec = {k: z[k] for k in z.files}
    rec["circuit"] = str(rec["circuit"])
    rec["n"] = int(rec["n"])
    rec["is_subcircuit"] = int(rec["is_subcircuit"])
    rec["sampled"] = "final_samples" in rec
    return rec


def initial_state(rec):
    """Initial state of a fixture (|0...0> when none was stored)."""
    from subquokka_dev_b200 import circuits
    n = rec["n"]
    if rec["sampled"]:
        s = circuits.random_state(n, int(rec["init_seed"]))
        assert abs(s.sum() - rec["init_sum"]) < 1e-9, "numpy RNG stream changed"
        return s
    if rec["init"].size:
        return rec["init"]
    s = np.zeros(1 << n, np.complex128)
    s[0] = 1
    return s


def compare(rec, final):
    """max |delta amp| between a computed final state and the fixture."""
    if rec["sampled"]:
        st = int(rec["sample_stride"])
        d = np.abs(final[::st] - rec["final_samples"]).max()
        d = max(d, abs(np.vdot(final, final).real - rec["final_norm2"]))
        d = max(d, abs(final.sum() - rec["final_sum"]) / np.sqrt(final.size))
        w = (final * np.exp(1j * np.arange(final.size) * 1e-3)).sum()
        d = max(d, abs(w - rec["final_wsum"]) / np.sqrt(final.size))
        return d
    return np.abs(final - rec["final"]).max()
