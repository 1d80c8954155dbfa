"""The `_C` drop-in surface (src/braket/snuqs/csrc/pymodule.cc:66-210) without
a GPU: names, constructor signatures, buffer protocols, modifiers."""
import numpy as np
import pytest

import oracle
from snuqs_b200 import _C

G = _C.operation.gate_operations
REF_BOUND = [  # pymodule.cc:88-120
    "Identity", "Hadamard", "PauliX", "PauliY", "PauliZ", "CX", "CY", "CZ", "S", "Si", "T",
    "Ti", "V", "Vi", "PhaseShift", "CPhaseShift", "CPhaseShift00", "CPhaseShift01",
    "CPhaseShift10", "RotX", "RotY", "RotZ", "Swap", "ISwap", "PSwap", "XY", "XX", "YY", "ZZ",
    "CCNot", "CSwap", "U", "GPhase"]


def make(name, targets, angles=(0.4, 1.2, -0.7), **kw):
    na = oracle.gate_num_angles(name)
    cls = getattr(G, name)
    if na == 3:
        return cls(targets, *angles[:3], **kw)
    if na == 2:
        return cls(targets, *angles[:2], **kw)
    if na == 1:
        return cls(targets, angles[0], **kw)
    return cls(targets, **kw)


def test_submodules_and_classes():
    for sub in ["operation", "functionals", "result_types", "stream", "event", "core"]:
        assert hasattr(_C, sub)
    for name in REF_BOUND + ["ECR", "CV", "PRx", "Unitary"]:
        assert issubclass(getattr(G, name), _C.operation.GateOperation)
    for f in ["apply", "initialize_zero", "initialize_basis_z"]:
        assert hasattr(_C.functionals, f)
    for f in ["mem_info", "device_count", "get_device", "set_device", "device_synchronize"]:
        assert hasattr(_C.core.cuda, f)
    assert _C.DeviceType.CUDA != _C.DeviceType.CPU


@pytest.mark.parametrize("name", REF_BOUND)
def test_gate_buffers_equal_reference_matrices(name):
    k = oracle.gate_qubits(name)
    g = make(name, list(range(k)))
    na = oracle.gate_num_angles(name)
    assert np.array_equal(np.array(g), oracle.ref_gate_matrix(name, (0.4, 1.2, -0.7)[:na]))
    assert g.targets == list(range(k))
    assert g.sliceable() is False


def test_ctrl_and_power_modifiers():
    x = np.array(G.PauliX([3, 1], ctrl_modifiers=[1]))
    assert np.array_equal(x.real, oracle.gate_matrix("CX").real)
    neg = np.array(G.PauliX([3, 1], ctrl_modifiers=[0]))
    want = np.eye(4)
    want[:2, :2] = [[0, 1], [1, 0]]
    assert np.array_equal(neg.real, want)
    inv = np.array(G.T([0], power=-1))
    assert np.allclose(inv, oracle.gate_matrix("Ti"))
    sq = np.array(G.V([0], power=2))
    assert np.allclose(sq, oracle.gate_matrix("PauliX"))
    with pytest.raises(ValueError):
        G.CX([0])  # wrong target count


def test_unitary_and_repr_eq():
    u = np.array([[0, 1], [1, 0]], dtype=complex)
    g = G.Unitary([2], u)
    assert np.array_equal(np.array(g), u)
    assert repr(G.RotX([1], 0.5)).startswith("RotX(0.5) {1}")
    assert G.RotX([1], 0.5) == G.RotX([1], 0.5)
    assert not (G.RotX([1], 0.5) == G.RotX([1], 0.6))


def test_cpu_state_vector_buffer_and_slice():
    sv = _C.result_types.StateVector(4)
    _C.functionals.initialize_basis_z(sv)
    a = np.array(sv, copy=False)
    assert a.shape == (16,) and a[0] == 1 and np.all(a[1:] == 0)
    sl = sv.slice(2, 1)
    assert np.array(sl, copy=False).shape == (4,)
    assert sv.num_elems() == 16
    assert "CPU" in repr(sv)


def test_apply_to_cpu_state_raises():
    sv = _C.result_types.StateVector(3)
    with pytest.raises(RuntimeError):
        _C.functionals.apply(sv, G.Hadamard([0]), 3, [0])
