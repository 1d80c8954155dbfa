"""The reference's own calling sequence through the `_C` drop-in
(src/braket/snuqs/simulation.py:113-122, 274-284, 197-206): StateVector on
CUDA, initialize_basis_z, one functionals.apply per gate, sync, cpu()."""
import numpy as np
import pytest

import oracle
from snuqs_b200 import _C, circuits

pytestmark = pytest.mark.gpu
G = _C.operation.gate_operations


def build(op):
    name, q, a = op[0], list(op[1]), op[2]
    if name == "Unitary":
        return G.Unitary(q, op[3])
    return getattr(G, name)(q, *a)


@pytest.fixture(scope="module", autouse=True)
def _gpu(cuda_required):
    yield


def simulate(ops, n, precision="complex128"):
    sv = _C.result_types.StateVector(_C.DeviceType.CUDA, n, precision)
    _C.functionals.initialize_basis_z(sv)
    gops = [build(op) for op in ops]
    for g in gops:
        _C.functionals.apply(sv, g, n, g.targets)
    sv.sync()
    return np.array(sv.cpu(), copy=True)


def test_reference_calling_sequence(golden_circuits):
    for key, (n, ops, ref) in golden_circuits.items():
        assert np.abs(simulate(ops, n) - ref).max() <= 1e-12, key


def test_random_33_gate_mix_14q():
    ops = circuits.random_all_gates(14, 400, seed=21)
    assert np.abs(simulate(ops, 14) - oracle.run_ops(ops, 14)).max() <= 1e-12


def test_modifiers_are_applied():
    n = 5
    sv = _C.result_types.StateVector(_C.DeviceType.CUDA, n)
    _C.functionals.initialize_basis_z(sv)
    ops = [G.Hadamard([0]), G.PauliX([0, 3], ctrl_modifiers=[1]),
           G.RotY([4, 1, 2], 0.7, ctrl_modifiers=[0, 1]), G.T([3], power=-1),
           G.V([2], power=2)]
    for g in ops:
        _C.functionals.apply(sv, g, n, g.targets)
    got = np.array(sv.cpu(), copy=True)
    ref = oracle.basis_state(n)
    for g in ops:
        oracle.apply_matrix(ref, n, np.array(g), list(g.targets))
    assert np.abs(got - ref).max() <= 1e-12


def test_copy_and_streams():
    n = 8
    s = _C.stream.Stream.create_nonblocking()
    sv = _C.result_types.StateVector(_C.DeviceType.CUDA, n)
    _C.functionals.initialize_basis_z(sv, stream=s)
    for q in range(n):
        g = G.Hadamard([q])
        _C.functionals.apply(sv, g, n, g.targets, stream=s)
    host = _C.result_types.StateVector(n, True)
    host.copy(sv, stream=s)
    a = np.array(host, copy=False)
    assert np.allclose(a, np.full(1 << n, 2 ** (-n / 2)), atol=1e-14)
    sv2 = host.cuda(stream=s)
    back = np.array(sv2.cpu(stream=s), copy=True)
    assert np.array_equal(back, a)
    e = _C.event.Event.create()
    e.record(s)
    e.synchronize()


def test_core_cuda_queries():
    assert _C.core.cuda.device_count() >= 1
    free, total = _C.core.cuda.mem_info()
    assert 0 < free <= total
    _C.core.cuda.device_synchronize()
