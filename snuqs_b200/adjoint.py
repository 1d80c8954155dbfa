"""Expectation values and their gradients on the engine.

* ``adjoint_gradient`` -- one forward pass plus one fused reverse (adjoint)
  pass (``sq_adjoint_gradient``): the energy and every parameter's gradient.
* ``parameter_shift_gradient`` -- the same gradient from 2 shifted forward
  evaluations per parametrised angle, on the same engine (the comparison the
  adjoint method is measured against).
* ``AdjointExpectation`` -- a ``torch.autograd.Function``: forward returns
  <H>(theta), backward returns the adjoint gradient.

A circuit is a list of ops ``(name, qubits, angles, params[, scales])`` or
``("Unitary", qubits, (), matrix)``; ``params[j]`` is the index of the
parameter angle ``j`` follows (-1 = constant), and ``angles[j]`` is filled
from ``theta[params[j]] * scales[j]`` by ``bind``.
"""
from __future__ import annotations

import ctypes
from typing import Sequence

import numpy as np

from . import capi

# Gates whose angles enter as exp(-i a G) with G of eigenvalue gap 1, so that
# dE/da = (E(a + pi/2) - E(a - pi/2)) / 2 holds exactly.
SHIFT_RULE_GATES = {"RotX", "RotY", "RotZ", "PhaseShift", "CPhaseShift", "CPhaseShift00",
                    "CPhaseShift01", "CPhaseShift10", "XX", "YY", "ZZ", "PSwap", "GPhase", "U"}


def bind(ops, theta: Sequence[float]):
    """Ops with every parametrised angle set to theta[param] * scale."""
    out = []
    for op in ops:
        if op[0] == "Unitary" or len(op) < 4:
            out.append(op)
            continue
        angles = list(op[2])
        scales = op[4] if len(op) > 4 else (1.0,) * len(angles)
        for j, p in enumerate(op[3]):
            if p >= 0:
                angles[j] = float(theta[p]) * scales[j]
        out.append((op[0], op[1], tuple(angles)) + tuple(op[3:]))
    return out


class Workspace:
    """The two work states the adjoint pass needs (psi and lambda = H psi)."""

    def __init__(self, n: int, dtype: int = capi.SQ_C128, stream=None):
        self.psi = capi.State(n, dtype, stream)
        self.lam = capi.State(n, dtype, stream)
        self.n, self.dtype, self.stream = n, dtype, stream

    def close(self):
        self.psi.close()
        self.lam.close()


def adjoint_gradient(ws: Workspace, ops, theta, terms, n_params: int):
    """(energy, gradient[n_params]) at theta for H = sum w P (terms = [(w, P)])."""
    bound = bind(ops, theta)
    arr, keep = capi.circuit_ops(bound)
    flat = "".join(p for _, p in terms).encode()
    w = np.ascontiguousarray([x for x, _ in terms] or [0.0], dtype=np.float64)
    e = ctypes.c_double(0)
    g = np.zeros(max(1, n_params), dtype=np.float64)
    capi.check(capi.lib().sq_adjoint_gradient(
        ws.psi.h, ws.lam.h, ctypes.cast(arr, ctypes.c_void_p), len(bound), flat,
        w.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), len(terms), n_params,
        ctypes.byref(e), g.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ws.stream))
    del keep
    return e.value, g[:n_params]


def energy(state: capi.State, ops, theta, terms) -> float:
    """<H> at theta, by a forward pass on `state`."""
    state.init_basis(0)
    state.apply_ops([op[:3] if op[0] != "Unitary" else op for op in bind(ops, theta)])
    return state.expectation(terms)


def parameter_shift_gradient(state: capi.State, ops, theta, terms, n_params: int,
                             max_evals: int | None = None):
    """Gradient by the two-term shift rule, one (+, -) pair per parametrised
    angle occurrence.  With max_evals, stops after that many circuit
    evaluations and returns (partial gradient, evaluations done)."""
    grad = np.zeros(n_params)
    evals = 0
    for i, op in enumerate(ops):
        if op[0] == "Unitary" or len(op) < 4:
            continue
        if op[0] not in SHIFT_RULE_GATES:
            raise ValueError(f"no two-term shift rule for {op[0]}")
        scales = op[4] if len(op) > 4 else (1.0,) * len(op[2])
        for j, p in enumerate(op[3]):
            if p < 0:
                continue
            vals = []
            for sgn in (+1, -1):
                shifted = list(bind(ops, theta))
                a = list(shifted[i][2])
                a[j] += sgn * np.pi / 2
                shifted[i] = (shifted[i][0], shifted[i][1], tuple(a))
                state.init_basis(0)
                state.apply_ops([o[:3] if o[0] != "Unitary" else o for o in shifted])
                vals.append(state.expectation(terms))
                evals += 1
            grad[p] += 0.5 * (vals[0] - vals[1]) * scales[j]
            if max_evals is not None and evals >= max_evals:
                return grad, evals
    return (grad, evals) if max_evals is not None else grad


def count_shift_evaluations(ops) -> int:
    """Circuit evaluations one parameter-shift gradient needs."""
    return 2 * sum(sum(1 for p in op[3] if p >= 0) for op in ops
                   if op[0] != "Unitary" and len(op) >= 4)


try:  # torch is plumbing here; the engine does not need it
    import torch

    class AdjointExpectation(torch.autograd.Function):
        """E(theta) = <0|U(theta)^dagger H U(theta)|0> with the adjoint
        gradient as its backward.  Usage:
        AdjointExpectation.apply(theta, workspace, ops, terms)."""

        @staticmethod
        def forward(ctx, theta, ws, ops, terms):
            th = theta.detach().cpu().numpy().astype(np.float64)
            e, g = adjoint_gradient(ws, ops, th, terms, th.size)
            ctx.save_for_backward(torch.from_numpy(g).to(theta.dtype))
            return theta.new_tensor(e)

        @staticmethod
        def backward(ctx, grad_out):
            (g,) = ctx.saved_tensors
            return grad_out * g.to(grad_out.device), None, None, None
except ImportError:  # pragma: no cover
    pass
