"""Parity of the CUDA engine against the oracle, through the C ABI.

complex128: max-abs amplitude error <= 1e-12 against the reference's own CPU
path (golden fixtures / oracle/_ref) and its C restatement.
complex64: max-abs <= 1e-5 and 1 - fidelity <= 1e-9 against the complex128
oracle (FP32 arithmetic, FP64 reductions)."""
import os

import numpy as np
import pytest

import oracle
from snuqs_b200 import capi, circuits
from tests.conftest import GOLDEN

pytestmark = pytest.mark.gpu
TOL128 = 1e-12
TOL64 = 1e-5


@pytest.fixture(scope="module", autouse=True)
def _gpu(cuda_required):
    import torch

    torch.cuda.init()
    yield


def run_engine(ops, n, dtype=capi.SQ_C128, fusion=True, tile_bits=12, reorder=True, psi0=None):
    st = capi.State(n, dtype)
    st.set_option(capi.SQ_OPT_FUSION, int(fusion))
    st.set_option(capi.SQ_OPT_TILE_BITS, tile_bits)
    st.set_option(capi.SQ_OPT_REORDER, int(reorder))
    if psi0 is None:
        st.init_basis(0)
    else:
        st.from_host(psi0)
    st.apply_ops(ops)
    out = st.to_host()
    st.close()
    return out


def fid_loss(a, b):
    a = a.astype(np.complex128)
    return 1.0 - abs(np.vdot(a, b)) ** 2 / (np.vdot(a, a).real * np.vdot(b, b).real)


@pytest.mark.parametrize("fusion", [True, False])
def test_every_gate_every_target_tuple(fusion):
    g = np.load(os.path.join(GOLDEN, "per_gate.npz"))
    ang = np.load(os.path.join(GOLDEN, "gate_matrices.npz"))["angles"]
    psi0 = g["psi0"]
    worst = 0.0
    for key in g.files:
        if key == "psi0":
            continue
        name, t = key.split("|")
        q = tuple(int(x) for x in t.split(",")) if t else ()
        na = oracle.gate_num_angles(name)
        out = run_engine([(name, q, tuple(ang[:na]))], 5, fusion=fusion, psi0=psi0)
        worst = max(worst, np.abs(out - g[key]).max())
    assert worst <= TOL128


@pytest.mark.parametrize("name", ["ECR", "CV", "PRx"])
def test_gates_the_reference_lacks(name):
    rng = np.random.default_rng(4)
    n = 6
    psi0 = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    k, na = oracle.gate_qubits(name), oracle.gate_num_angles(name)
    for _ in range(6):
        q = tuple(int(x) for x in rng.choice(n, size=k, replace=False))
        a = tuple(rng.uniform(0, 2 * np.pi, size=na))
        ref = oracle.run_ops([(name, q, a)], n, state=psi0)
        assert np.abs(run_engine([(name, q, a)], n, psi0=psi0) - ref).max() <= TOL128


@pytest.mark.parametrize("fusion", [True, False])
def test_golden_circuits(golden_circuits, fusion):
    for key, (n, ops, ref) in golden_circuits.items():
        out = run_engine(ops, n, fusion=fusion)
        assert np.abs(out - ref).max() <= TOL128, key


def test_ghz20_known_answer():
    out = run_engine(circuits.ghz(20), 20)
    want = np.zeros(1 << 20, dtype=np.complex128)
    want[0] = want[-1] = np.sqrt(0.5)
    assert np.abs(out - want).max() <= TOL128


@pytest.mark.parametrize("n", [4, 6, 9, 12, 13, 16, 18])
def test_random_all_gates(n):
    ops = circuits.random_all_gates(n, 300, seed=100 + n)
    ref = oracle.run_ops(ops, n)
    for tb, reorder in [(12, True), (9, False), (10, True)]:
        out = run_engine(ops, n, tile_bits=tb, reorder=reorder)
        assert np.abs(out - ref).max() <= TOL128, (n, tb, reorder)


def test_workload_mix_20q_400_gates():
    ops = circuits.random_mix(20, 400, seed=1234)
    ref = oracle.run_ops(ops, 20)
    assert np.abs(run_engine(ops, 20) - ref).max() <= TOL128
    assert np.abs(run_engine(ops, 20, fusion=False) - ref).max() <= TOL128


def test_quantum_volume_unitaries_16q():
    ops = circuits.quantum_volume(16, 16, seed=3)
    ref = oracle.run_ops(ops, 16)
    assert np.abs(run_engine(ops, 16) - ref).max() <= TOL128


def test_large_and_controlled_unitaries():
    rng = np.random.default_rng(5)
    n = 12
    st = capi.State(n)
    st.init_basis(3)
    ref = oracle.basis_state(n, 3)
    for i in range(30):
        k = int(rng.integers(1, 7))  # k = 5, 6 run unfused
        qs = [int(x) for x in rng.choice(n, size=k + 2, replace=False)]
        u = circuits.haar_unitary(1 << k, rng)
        nc = int(rng.integers(0, 3))
        c, v = qs[k:k + nc], [int(x) for x in rng.integers(0, 2, size=nc)]
        st.apply_matrix(u, qs[:k], c, v)
        D = 1 << (nc + k)
        full = np.eye(D, dtype=np.complex128)
        blk = (int("".join(map(str, v)), 2) if nc else 0) << k
        full[blk:blk + (1 << k), blk:blk + (1 << k)] = u
        oracle.apply_matrix(ref, n, full, c + qs[:k])
    assert np.abs(st.to_host() - ref).max() <= TOL128


def test_complex64_against_complex128_oracle():
    for n, ops in [(16, circuits.random_mix(16, 400, seed=8)),
                   (14, circuits.quantum_volume(14, 14, seed=2)),
                   (12, circuits.random_all_gates(12, 300, seed=6))]:
        ref = oracle.run_ops(ops, n)
        out = run_engine(ops, n, dtype=capi.SQ_C64)
        assert out.dtype == np.complex64
        assert np.abs(out - ref).max() <= TOL64, n
        assert fid_loss(out, ref) <= 1e-9, n


def test_reductions():
    rng = np.random.default_rng(12)
    for dtype, tol in [(capi.SQ_C128, 1e-12), (capi.SQ_C64, 1e-5)]:
        for n in [5, 10, 17]:
            ops = circuits.random_mix(n, 150, seed=n)
            ref = oracle.run_ops(ops, n)
            st = capi.State(n, dtype)
            st.init_basis(0)
            st.apply_ops(ops)
            terms = circuits.random_pauli_hamiltonian(n, 40, seed=n)
            terms += [(0.5, "Z" * n), (-1.25, "I" * n), (0.75, "Y" * n)]
            want = oracle.expectation(ref, n, terms)
            assert abs(st.expectation(terms) - want) <= tol * max(1.0, abs(want)), (n, dtype)
            assert abs(st.norm2() - 1.0) <= tol
            import torch

            probs = torch.empty(1 << n, dtype=torch.float64, device="cuda")
            capi.check(capi.lib().sq_probabilities(st.h, probs.data_ptr(), None))
            torch.cuda.synchronize()
            assert np.abs(probs.cpu().numpy() - oracle.probabilities(ref)).max() <= tol
            st.close()


def test_apply_gate_buffer_is_cu_applygate():
    """sq_apply_gate_buffer replaces cu::applyGate(buffer, gate, targets,
    nqubits, nelems) with a device matrix, unqueued."""
    import ctypes
    import torch

    n = 11
    rng = np.random.default_rng(2)
    psi0 = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    buf = torch.from_numpy(psi0.copy()).cuda()
    ref = psi0.copy()
    for name in ["Hadamard", "CX", "CCNot", "U", "XY", "GPhase"]:
        k, na = oracle.gate_qubits(name), oracle.gate_num_angles(name)
        q = [int(x) for x in rng.choice(n, size=k, replace=False)]
        a = tuple(rng.uniform(0, 6, size=na))
        m = oracle.gate_matrix(name, a)
        dm = torch.from_numpy(m.copy()).cuda()
        t = (ctypes.c_uint64 * max(1, k))(*q)
        capi.check(capi.lib().sq_apply_gate_buffer(buf.data_ptr(), dm.data_ptr(), t, k, n,
                                                   1 << n, None))
        oracle.apply_matrix(ref, n, m, q)
    torch.cuda.synchronize()
    assert np.abs(buf.cpu().numpy() - ref).max() <= TOL128


def test_invalid_arguments_raise_not_exit():
    st = capi.State(4)
    with pytest.raises(capi.SqError) as e:
        st.apply_gate("CX", (1, 1))
    assert e.value.status == capi.SQ_ERR_INVALID
    with pytest.raises(capi.SqError):
        st.apply_gate("Hadamard", (4,))
    with pytest.raises(capi.SqError):
        st.init_basis(16)
    st.close()


def test_fused_equals_unfused_at_26_qubits_64bit_indices():
    """Fused sweeps vs the unfused per-gate kernels on the same GPU, and a
    forward-then-inverse round trip back to |0>."""
    n = 26
    ops = circuits.random_mix(n, 120, seed=77)
    a = run_engine(ops, n)
    b = run_engine(ops, n, fusion=False)
    assert np.abs(a - b).max() <= TOL128
    assert abs(np.vdot(a, a).real - 1.0) <= 1e-12


def test_quantum_volume_28_qubits_fused_unfused_and_complex64():
    """The QV-28 configuration (depth 28, 392 Haar 4x4 Unitary gates): fused
    sweeps against the unfused per-gate kernels (complex128), and the
    complex64 state against the complex128 one (1 - fidelity)."""
    n = 28
    ops = circuits.quantum_volume(n, n, seed=28)
    a = run_engine(ops, n)
    b = run_engine(ops, n, fusion=False)
    assert np.abs(a - b).max() <= TOL128
    c = run_engine(ops, n, dtype=capi.SQ_C64)
    assert fid_loss(c, a) <= 1e-9
    assert np.abs(c - a).max() <= TOL64
