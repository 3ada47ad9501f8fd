"""torch.autograd bridge over the adjoint sweep (qk_adjoint_grad).

``ParamCircuit`` is a circuit template whose RX/RY/RZ gates may read their
angle from a parameter vector; ``expectation(params, pc, terms)`` returns
<H> as a differentiable torch scalar.  One call runs the forward pass, the
adjoint backward sweep and keeps the gradient for autograd's backward, so a
parameter update costs one engine call.  U3(theta, phi, lambda) enters as
RZ(lambda) RY(theta) RZ(phi) (equal up to a global phase, which no
expectation value sees).
"""
from __future__ import annotations

import numpy as np
import torch

from .engine import Circuit, StateVector, adjoint_grad, make_gate


class ParamCircuit:
    """Gate template: entries (name, qubits, angle_or_param, coeff)."""

    def __init__(self, nqubits: int):
        self.n = int(nqubits)
        self.ops = []          # (name, qubits, value, param index or -1, coeff)
        self.nparams = 0

    def param(self) -> int:
        self.nparams += 1
        return self.nparams - 1

    def rot(self, name: str, q: int, p: int):
        assert name in ("RX", "RY", "RZ")
        self.ops.append((name, [q], 0.0, int(p), None))

    def fixed(self, name: str, qubits, value: float = 0.0, coeff=None):
        self.ops.append((name, list(qubits), float(value), -1, coeff))

    def u3(self, q: int, p_theta: int, p_phi: int, p_lambda: int):
        self.rot("RZ", q, p_lambda)
        self.rot("RY", q, p_theta)
        self.rot("RZ", q, p_phi)

    def state(self, dtype: str) -> StateVector:
        """This circuit's device state in `dtype`, reset to |0...0>: kept between
        calls together with its adjoint workspace; `close` frees them."""
        states = self.__dict__.setdefault("_states", {})
        sv = states.get(dtype)
        if sv is None:
            sv = states[dtype] = StateVector(self.n, dtype)
        sv.reset()
        return sv

    def close(self) -> None:
        for sv in self.__dict__.pop("_states", {}).values():
            sv.close()

    def bind(self, params: np.ndarray):
        """(Circuit with the parameter values in place, param_index array)."""
        gates, idx = [], []
        for name, qs, val, p, coeff in self.ops:
            angle = float(params[p]) if p >= 0 else val
            gates.append(make_gate(name, qs, angle, coeff))
            idx.append(p)
        return Circuit(gates), np.asarray(idx, dtype=np.int32)


class _Expectation(torch.autograd.Function):
    @staticmethod
    def forward(ctx, params, pc, terms, dtype, checkpoints, fused):
        p = params.detach().to("cpu", torch.float64).numpy()
        circ, idx = pc.bind(p)
        sv = pc.state(dtype)
        ev, grad, drift = adjoint_grad(sv, circ, idx, pc.nparams, terms, checkpoints, fused)
        ctx.save_for_backward(torch.as_tensor(grad, dtype=params.dtype, device=params.device))
        ctx.drift = drift
        return torch.tensor(ev, dtype=params.dtype, device=params.device)

    @staticmethod
    def backward(ctx, g):
        (grad,) = ctx.saved_tensors
        return g * grad, None, None, None, None, None


def expectation(params: torch.Tensor, pc: ParamCircuit, terms, dtype: str = "c128", checkpoints: int = -1,
                fused: bool = True):
    """<0| U(params)^dag H U(params) |0> as a differentiable torch scalar."""
    return _Expectation.apply(params, pc, terms, dtype, checkpoints, fused)


def hea_template(n: int, layers: int) -> ParamCircuit:
    """The hardware-efficient ansatz of the variational workloads: per layer
    RY and RZ on every qubit (one parameter each) and a CNOT ladder written as
    U2 in the reference's big-endian order."""
    from .circuits import CNOT_BIG_ENDIAN
    pc = ParamCircuit(n)
    for _ in range(layers):
        for q in range(n):
            pc.rot("RY", q, pc.param())
            pc.rot("RZ", q, pc.param())
        for q in range(n - 1):
            pc.fixed("U2", [q, q + 1], coeff=CNOT_BIG_ENDIAN)
    return pc
