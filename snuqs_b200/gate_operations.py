"""Gate operations for the Braket front ends, with the gates and modifiers
the reference drops.

The reference's JAQCD table (src/braket/snuqs/gate_operations.py:206-239)
lists CV, ECR and PRx as removed, and its `Unitary` (:23-39) calls the
_C GateOperation constructor with keywords it does not accept, so every
Unitary instruction raises.  Its OpenQASM front end folds inv / pow / ctrl /
negctrl into (ctrl_modifiers, power) (src/braket/snuqs/openqasm/
program_context.py:744-781) and hands them to GateOperation, which stores and
ignores them (operation.cc:96-109).

Here:
* `BRAKET_GATES` maps every Braket gate name, CV / ECR / PRx / Unitary
  included, to its `_C.operation.gate_operations` class;
* `Unitary(targets, matrix, ctrl_modifiers, power)` works;
* `fold_modifiers` restates the OpenQASM modifier folding (inv flips the
  power's sign, pow multiplies it, ctrl adds control value 1 and negctrl
  control value 0 per argument count);
* `gate_operation(name, targets, params, ctrl_modifiers, power)` builds the
  operation exactly as program_context.add_gate_instruction would, and the
  engine applies the modifiers: integer powers in `_C`, fractional powers
  here by the principal branch of the matrix power (U^p = V diag(l^p) V^H for
  the eigendecomposition U = V diag(l) V^H), controls as controlled gates.
The JAQCD instruction translators are registered when the Braket SDK is
importable.
"""
from __future__ import annotations

from typing import Sequence

import numpy as np

from ._C.operation import gate_operations as _G

BRAKET_GATES = {
    "i": _G.Identity, "h": _G.Hadamard, "x": _G.PauliX, "y": _G.PauliY, "z": _G.PauliZ,
    "cnot": _G.CX, "cy": _G.CY, "cz": _G.CZ, "s": _G.S, "si": _G.Si, "t": _G.T, "ti": _G.Ti,
    "v": _G.V, "vi": _G.Vi, "phaseshift": _G.PhaseShift, "cphaseshift": _G.CPhaseShift,
    "cphaseshift00": _G.CPhaseShift00, "cphaseshift01": _G.CPhaseShift01,
    "cphaseshift10": _G.CPhaseShift10, "rx": _G.RotX, "ry": _G.RotY, "rz": _G.RotZ,
    "swap": _G.Swap, "iswap": _G.ISwap, "pswap": _G.PSwap, "xy": _G.XY, "xx": _G.XX,
    "yy": _G.YY, "zz": _G.ZZ, "ccnot": _G.CCNot, "cswap": _G.CSwap, "U": _G.U,
    "gphase": _G.GPhase, "cv": _G.CV, "ecr": _G.ECR, "prx": _G.PRx, "unitary": _G.Unitary,
}


def Unitary(targets: Sequence[int], matrix, ctrl_modifiers: Sequence[int] = (), power: float = 1):
    """A Unitary gate operation (what the reference's Unitary intends)."""
    m = np.array(matrix, dtype=np.complex128)
    k = len(targets) - len(ctrl_modifiers)
    if k < 0 or m.shape != (1 << k, 1 << k):
        raise ValueError(f"a Unitary on {k} target qubits needs a {1 << max(k, 0)}x{1 << max(k, 0)} matrix")
    if not np.allclose(m @ m.conj().T, np.eye(1 << k), atol=1e-10):
        raise ValueError("matrix is not unitary")
    ctrl = [int(c) for c in ctrl_modifiers]
    if float(power).is_integer():
        return _G.Unitary(list(targets), m, ctrl_modifiers=ctrl, power=float(power))
    return _G.Unitary(list(targets), matrix_power(m, power), ctrl_modifiers=ctrl, power=1.0)


def fold_modifiers(modifiers: Sequence[tuple[str, int | float | None]]) -> tuple[list[int], float]:
    """(ctrl_modifiers, power) of an OpenQASM modifier list, e.g.
    [("ctrl", 1), ("pow", 0.5), ("inv", None), ("negctrl", 2)]."""
    power: float = 1
    if sum(1 for m, _ in modifiers if m == "inv") % 2:
        power *= -1
    ctrl: list[int] = []
    for m, arg in modifiers:
        if m in ("ctrl", "negctrl"):
            ctrl += [1 if m == "ctrl" else 0] * int(1 if arg is None else arg)
        elif m == "pow":
            power *= arg
        elif m != "inv":
            raise ValueError(f"unknown gate modifier {m!r}")
    return ctrl, power


def matrix_power(m: np.ndarray, power: float) -> np.ndarray:
    """Principal-branch power of a unitary matrix."""
    if float(power).is_integer():
        p = int(power)
        base = m if p >= 0 else m.conj().T
        return np.linalg.matrix_power(base, abs(p))
    w, v = np.linalg.eig(m)
    # A unitary is normal: orthonormalise its eigenvectors (QR keeps each
    # eigenspace) so that V^-1 = V^H.
    v, _ = np.linalg.qr(v)
    w = np.diag(v.conj().T @ m @ v)
    return (v * np.exp(1j * power * np.angle(w)) * np.abs(w) ** power) @ v.conj().T


def gate_operation(name: str, targets: Sequence[int], params: Sequence[float] = (),
                   ctrl_modifiers: Sequence[int] = (), power: float = 1):
    """The operation program_context.add_gate_instruction builds for a gate
    with modifiers; targets list the control qubits first (Braket order)."""
    key = name if name in BRAKET_GATES else name.lower()
    if key not in BRAKET_GATES:
        raise ValueError(f"unknown gate {name!r}")
    cls = BRAKET_GATES[key]
    targets = [int(t) for t in targets]
    ctrl = [int(c) for c in ctrl_modifiers]
    if float(power).is_integer():
        return cls(targets, *params, ctrl_modifiers=ctrl, power=float(power))
    # Fractional power: the base gate's matrix raised here, controls kept.
    nc = len(ctrl)
    base = cls(targets[nc:], *params)
    m = np.array(base, copy=True)
    return _G.Unitary(targets, matrix_power(m, power), ctrl_modifiers=ctrl, power=1.0)


try:  # JAQCD instruction translators, when the Braket SDK is present
    from functools import singledispatch

    import braket.ir.jaqcd as _ji

    @singledispatch
    def from_braket_instruction(instruction):
        raise NotImplementedError(f"Instruction {instruction} not recognized")

    def _reg(ir_cls, fn):
        from_braket_instruction.register(ir_cls)(fn)

    for _name, _ir in [("i", "I"), ("h", "H"), ("x", "X"), ("y", "Y"), ("z", "Z"), ("s", "S"),
                       ("si", "Si"), ("t", "T"), ("ti", "Ti"), ("v", "V"), ("vi", "Vi")]:
        if hasattr(_ji, _ir):
            _reg(getattr(_ji, _ir), lambda ins, _n=_name: BRAKET_GATES[_n]([ins.target]))
    for _name, _ir in [("rx", "Rx"), ("ry", "Ry"), ("rz", "Rz"), ("phaseshift", "PhaseShift")]:
        if hasattr(_ji, _ir):
            _reg(getattr(_ji, _ir), lambda ins, _n=_name: BRAKET_GATES[_n]([ins.target], ins.angle))
    for _name, _ir in [("cnot", "CNot"), ("cy", "CY"), ("cz", "CZ"), ("cv", "CV")]:
        if hasattr(_ji, _ir):
            _reg(getattr(_ji, _ir), lambda ins, _n=_name: BRAKET_GATES[_n]([ins.control, ins.target]))
    for _name, _ir in [("swap", "Swap"), ("iswap", "ISwap"), ("ecr", "ECR")]:
        if hasattr(_ji, _ir):
            _reg(getattr(_ji, _ir), lambda ins, _n=_name: BRAKET_GATES[_n](list(ins.targets)))
    for _name, _ir in [("pswap", "PSwap"), ("xy", "XY"), ("xx", "XX"), ("yy", "YY"), ("zz", "ZZ")]:
        if hasattr(_ji, _ir):
            _reg(getattr(_ji, _ir), lambda ins, _n=_name: BRAKET_GATES[_n](list(ins.targets), ins.angle))
    for _name, _ir in [("cphaseshift", "CPhaseShift"), ("cphaseshift00", "CPhaseShift00"),
                       ("cphaseshift01", "CPhaseShift01"), ("cphaseshift10", "CPhaseShift10")]:
        if hasattr(_ji, _ir):
            _reg(getattr(_ji, _ir),
                 lambda ins, _n=_name: BRAKET_GATES[_n]([ins.control, ins.target], ins.angle))
    if hasattr(_ji, "CCNot"):
        _reg(_ji.CCNot, lambda ins: _G.CCNot([*ins.controls, ins.target]))
    if hasattr(_ji, "CSwap"):
        _reg(_ji.CSwap, lambda ins: _G.CSwap([ins.control, *ins.targets]))
    if hasattr(_ji, "Unitary"):
        _reg(_ji.Unitary, lambda ins: Unitary(
            list(ins.targets), np.array(ins.matrix)[..., 0] + 1j * np.array(ins.matrix)[..., 1]))
except Exception:  # noqa: BLE001 - the SDK is optional
    pass
