"""Front-end gate operations without a GPU: every Braket gate name resolves
(CV, ECR, PRx and Unitary included), OpenQASM modifiers fold as the
reference front end folds them, and powers / controls give the matrices of
their definitions."""
import numpy as np
import pytest
import scipy.linalg as sl

from snuqs_b200 import circuits
from snuqs_b200 import gate_operations as go


def controlled(m, ctrl):
    """Full matrix of `m` controlled on leading qubits with values ctrl."""
    k = int(m.shape[0]).bit_length() - 1
    nc = len(ctrl)
    d = 1 << (nc + k)
    full = np.eye(d, dtype=np.complex128)
    blk = int("".join(map(str, ctrl)), 2) << k if nc else 0
    full[blk:blk + (1 << k), blk:blk + (1 << k)] = m
    return full


def test_every_braket_gate_name_builds():
    for name, cls in go.BRAKET_GATES.items():
        if name == "unitary":
            continue
        nq = {"cnot": 2, "cy": 2, "cz": 2, "cphaseshift": 2, "cphaseshift00": 2, "cphaseshift01": 2,
              "cphaseshift10": 2, "swap": 2, "iswap": 2, "pswap": 2, "xy": 2, "xx": 2, "yy": 2, "zz": 2,
              "cv": 2, "ecr": 2, "ccnot": 3, "cswap": 3, "gphase": 0}.get(name, 1)
        nang = {"U": 3, "prx": 2}.get(name, 1 if name in ("phaseshift", "cphaseshift", "cphaseshift00",
                                                        "cphaseshift01", "cphaseshift10", "rx", "ry", "rz",
                                                        "pswap", "xy", "xx", "yy", "zz", "gphase") else 0)
        g = cls(list(range(nq)), *([0.3] * nang))
        m = np.array(g)
        assert m.shape == (1 << nq, 1 << nq)
        assert np.allclose(m @ m.conj().T, np.eye(1 << nq), atol=1e-12), name


def test_fold_modifiers_like_the_openqasm_front_end():
    assert go.fold_modifiers([]) == ([], 1)
    assert go.fold_modifiers([("inv", None)]) == ([], -1)
    assert go.fold_modifiers([("inv", None), ("inv", None)]) == ([], 1)
    assert go.fold_modifiers([("ctrl", 2), ("negctrl", 1), ("pow", 3)]) == ([1, 1, 0], 3)
    assert go.fold_modifiers([("pow", 0.5), ("inv", None)]) == ([], -0.5)
    with pytest.raises(ValueError):
        go.fold_modifiers([("twice", 2)])


@pytest.mark.parametrize("power", [1, 2, -1, 3, 0.5, -0.25, 1.5])
def test_powers_and_controls(power):
    rng = np.random.default_rng(int(abs(power) * 100))
    base = np.array(go.BRAKET_GATES["rx"]([0], 0.7))
    g = go.gate_operation("rx", [5, 2, 0], [0.7], ctrl_modifiers=[1, 0], power=power)
    want = controlled(sl.fractional_matrix_power(base, power) if not float(power).is_integer()
                      else np.linalg.matrix_power(base if power > 0 else base.conj().T, abs(int(power))),
                      [1, 0])
    assert np.abs(np.array(g) - want).max() <= 1e-12
    u = circuits.haar_unitary(4, rng)
    g = go.Unitary([3, 1, 4], u, ctrl_modifiers=[1], power=power)
    want = controlled(sl.fractional_matrix_power(u, power) if not float(power).is_integer()
                      else np.linalg.matrix_power(u if power > 0 else u.conj().T, abs(int(power))), [1])
    assert np.abs(np.array(g) - want).max() <= 1e-12


def test_unitary_validates_its_matrix():
    with pytest.raises(ValueError):
        go.Unitary([0, 1], np.eye(2))
    with pytest.raises(ValueError):
        go.Unitary([0], np.array([[1, 1], [0, 1]]))
    with pytest.raises(ValueError):
        go.gate_operation("nosuchgate", [0])
