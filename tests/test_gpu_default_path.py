"""The engine's DEFAULT path against the reference's own CPU gate path.

No option is overridden here: tiles of 2^11 amplitudes (complex128) / 2^12
(complex64) with 128-byte contiguous runs, the selecting planner (states of
>= 18 qubits), and JIT-specialised sweep kernels (states of >= 20 qubits).
That is the configuration the benchmark times.  The oracle is oracle/_ref:
the reference's cpu::applyGate (gate_operations_impl_cpu.cc:131-148) with the
reference's gate constructors (gate_operations.cc), compiled from the
reference sources; Unitary gates go through the same cpu::applyGate with the
caller's matrix.

complex128: max-abs amplitude error <= 1e-12.  complex64: max-abs <= 1e-5
and 1 - fidelity <= 1e-9 against the complex128 oracle.
"""
import numpy as np
import pytest

import oracle
from snuqs_b200 import capi, circuits

pytestmark = pytest.mark.gpu
TOL128 = 1e-12
TOL64 = 1e-5
FID64 = 1e-9


@pytest.fixture(scope="module", autouse=True)
def _gpu(cuda_required):
    import torch

    torch.cuda.init()
    yield


def host_ram_ok(n: int, copies: float) -> bool:
    """`copies` complex128 states of 2^n amplitudes fit in available host RAM."""
    import psutil

    return psutil.virtual_memory().available > copies * (1 << n) * 16


def device_ram_ok(n: int, amp_bytes: int, copies: float = 1.2) -> bool:
    import torch

    free, _ = torch.cuda.mem_get_info()
    return free > copies * (1 << n) * amp_bytes


def engine(ops, n, dtype=capi.SQ_C128, as_matrices=False, out=None):
    """Runs ops from |0...0> with default options; returns (state, launches,
    JIT sweep launches).  as_matrices: every gate as a dense matrix through
    sq_apply_matrix, the calling sequence of the benchmark and of the
    reference front end (GateOperation matrices)."""
    st = capi.State(n, dtype)
    st.init_basis(0)
    j0 = capi.jit_info()[1]
    if as_matrices:
        for op in ops:
            st.apply_matrix(circuits.op_matrix(op, capi.gate_matrix), op[1])
    else:
        st.apply_ops(ops)
    st.flush()
    launches = st.launches()
    psi = st.to_host(out)
    st.close()
    return psi, launches, capi.jit_info()[1] - j0


def max_abs_diff(a, b, chunk=1 << 24) -> float:
    worst = 0.0
    for i in range(0, a.size, chunk):
        d = a[i:i + chunk].astype(np.complex128) - b[i:i + chunk]
        worst = max(worst, float(np.abs(d).max()))
    return worst


def fidelity_loss(a, b, chunk=1 << 24) -> float:
    ab, aa, bb = 0j, 0.0, 0.0
    for i in range(0, a.size, chunk):
        x = a[i:i + chunk].astype(np.complex128)
        y = b[i:i + chunk]
        ab += np.vdot(x, y)
        aa += np.vdot(x, x).real
        bb += np.vdot(y, y).real
    return 1.0 - abs(ab) ** 2 / (aa * bb)


def reference(ops, n):
    return oracle.run_ops(ops, n, use_ref=True)


@pytest.mark.parametrize("n", [22, 24])
def test_random_mix_default_path(n):
    """The benchmark's generator (seed 1234, 400 gates) at 22 and 24 qubits,
    complex128 through named gates and through dense matrices, and
    complex64."""
    ops = circuits.random_mix(n, 400, seed=1234)
    ref = reference(ops, n)
    for as_m in (False, True):
        psi, launches, jit = engine(ops, n, as_matrices=as_m)
        assert jit > 0 and jit == launches, "the default path runs JIT sweeps"
        assert launches < len(ops) // 4, "the gates are fused"
        assert max_abs_diff(psi, ref) <= TOL128, (n, as_m)
    psi64, _, _ = engine(ops, n, dtype=capi.SQ_C64)
    assert psi64.dtype == np.complex64
    assert max_abs_diff(psi64, ref) <= TOL64
    assert fidelity_loss(psi64, ref) <= FID64


def test_every_gate_kind_22_qubits_default_path():
    """All 33 reference gates plus ECR/CV/PRx and 3-qubit gates on the
    extreme index bits, 22 qubits (JIT, selecting planner)."""
    n = 22
    ops = circuits.random_all_gates(n, 400, seed=2222)
    ops += [("CX", (0, n - 1), ()), ("CX", (n - 1, 0), ()), ("CCNot", (0, n - 1, n // 2), ()),
            ("CSwap", (n - 1, 0, 1), ()), ("Swap", (0, n - 1), ()), ("XX", (0, n - 1), (0.4,)),
            ("ECR", (3, n - 2), ()), ("CV", (n - 1, 5), ()), ("PRx", (7,), (0.3, 1.1))]
    ref = oracle.run_ops(ops, n)
    psi, launches, jit = engine(ops, n)
    assert jit == launches > 0
    assert max_abs_diff(psi, ref) <= TOL128


def test_quantum_volume_28_against_reference():
    """QV-28: depth 28, 392 Haar 4x4 Unitary gates on random pairs (4 GiB
    complex128 state), complex128 and complex64."""
    n = 28
    if not host_ram_ok(n, 3.5):
        pytest.skip("host RAM below 3.5 complex128 states of 28 qubits")
    ops = circuits.quantum_volume(n, n, seed=28)
    ref = reference(ops, n)
    psi, launches, jit = engine(ops, n)
    assert jit == launches > 0
    assert max_abs_diff(psi, ref) <= TOL128
    del psi
    psi64, _, _ = engine(ops, n, dtype=capi.SQ_C64)
    assert max_abs_diff(psi64, ref) <= TOL64
    assert fidelity_loss(psi64, ref) <= FID64


def test_headline_30q_random_mix_against_reference():
    """The benchmark's own workload: 30 qubits complex128, the 400-gate
    random mix (seed 1234), every gate as a dense matrix exactly as the
    benchmark submits it, against the reference CPU path on the host."""
    n = 30
    if not host_ram_ok(n, 2.3):
        pytest.skip("host RAM below 2.3 complex128 states of 30 qubits")
    if not device_ram_ok(n, 16):
        pytest.skip("device memory below 1.2 states of 30 qubits")
    ops = circuits.random_mix(n, 400, seed=1234)
    ref = reference(ops, n)
    out = np.empty(1 << n, dtype=np.complex128)
    psi, launches, jit = engine(ops, n, as_matrices=True, out=out)
    assert jit == launches > 0
    err = max_abs_diff(psi, ref)
    print(f"30q random mix: {launches} sweeps, max-abs {err:.3e}")
    assert err <= TOL128


def _round_trip(n, dtype, ngates, norm_tol, z_tol):
    ops = circuits.random_mix(n, ngates, seed=n)
    st = capi.State(n, dtype)
    st.init_basis(0)
    st.apply_ops(ops)
    st.flush()
    e_mid = st.norm2()
    for op in reversed(ops):
        m = circuits.op_matrix(op, oracle.gate_matrix)
        st.apply_matrix(m.conj().T, op[1])
    st.flush()
    assert abs(e_mid - 1.0) <= norm_tol
    assert abs(st.norm2() - 1.0) <= norm_tol
    assert abs(st.expectation([(1.0, "Z" * n)]) - 1.0) <= z_tol  # |0..0> has <Z..Z> = 1
    st.close()


def test_round_trip_32_qubits_400_gates():
    """32 qubits complex128 (64 GiB; beyond 32-bit indices): the 400-gate
    mix of the 32-qubit configuration, then its inverse, back to |0...0>."""
    if not device_ram_ok(32, 16, 1.05):
        pytest.skip("needs 68 GiB free device memory")
    _round_trip(32, capi.SQ_C128, 400, 1e-11, 1e-10)


def test_round_trip_33_qubits_complex64_400_gates():
    """33 qubits complex64 (64 GiB): 400 gates and their inverse."""
    if not device_ram_ok(33, 8, 1.05):
        pytest.skip("needs 68 GiB free device memory")
    _round_trip(33, capi.SQ_C64, 400, 1e-4, 1e-3)


@pytest.mark.parametrize("low_bits", [0, 4, 5])
def test_remapping_sweeps_against_reference(low_bits):
    """Qubit remapping on and off (SQ_OPT_REMAP), with the default and with
    longer contiguous runs: the same state as the reference CPU path, and
    the remapping plan uses fewer sweeps or as many."""
    n = 24
    for ops in (circuits.random_mix(n, 400, seed=24), circuits.quantum_volume(n, 12, seed=24)):
        ref = reference(ops, n)
        launches = {}
        for remap in (1, 0):
            st = capi.State(n)
            st.set_option(capi.SQ_OPT_REMAP, remap)
            if low_bits:
                st.set_option(capi.SQ_OPT_LOW_BITS, low_bits)
            st.init_basis(0)
            st.apply_ops(ops)
            st.flush()
            launches[remap] = st.launches()
            psi = st.to_host()
            st.close()
            assert max_abs_diff(psi, ref) <= TOL128, (low_bits, remap)
        assert launches[1] <= launches[0] + 1


def test_same_circuit_with_new_angles_on_one_state():
    """A state runs one gate sequence with three sets of angles (its plan is
    re-emitted from the sweep recipes after the first), each against the
    reference; then a different sequence (planned anew)."""
    n = 22
    rng = np.random.default_rng(5)
    st = capi.State(n)
    for k in range(3):
        ops = circuits.vqe_ansatz(n, rng.uniform(0, 2 * np.pi, 12 * n))
        st.init_basis(0)
        st.apply_ops(ops)
        st.flush()
        assert max_abs_diff(st.to_host(), reference(ops, n)) <= TOL128, k
    ops = circuits.random_mix(n, 200, seed=3)
    st.init_basis(0)
    st.apply_ops(ops)
    st.flush()
    assert max_abs_diff(st.to_host(), reference(ops, n)) <= TOL128
    st.close()
