"""Edge cases of the CUDA path against the oracle, through the C ABI: the
smallest states (1-3 qubits run unfused, 4 is the smallest fused tile), an
empty circuit, repeated and empty flushes, circuits of only diagonal or only
global-phase gates, every qubit of a state as a target, controls on the
highest and lowest index bits, and ragged batches (one circuit, circuits of 4
qubits, mixed sizes in one launch)."""
import numpy as np
import pytest

import oracle
from snuqs_b200 import capi, circuits

pytestmark = pytest.mark.gpu
TOL = 1e-12


@pytest.fixture(scope="module", autouse=True)
def _gpu(cuda_required):
    yield


def run(ops, n, dtype=capi.SQ_C128, jit=-1, psi0=None):
    st = capi.State(n, dtype)
    st.set_option(capi.SQ_OPT_JIT, jit)
    if psi0 is None:
        st.init_basis(0)
    else:
        st.from_host(psi0)
    st.apply_ops(ops)
    out = st.to_host()
    st.close()
    return out


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5])
def test_smallest_states(n):
    names = [g for g in circuits.REFERENCE_TEST_GATES if oracle.gate_qubits(g) <= n]
    ops = circuits.random_all_gates(n, 60, seed=n, names=names)
    assert np.abs(run(ops, n) - oracle.run_ops(ops, n)).max() <= TOL


@pytest.mark.parametrize("jit", [0, 1])
def test_empty_circuit_and_repeated_flushes(jit):
    n = 6
    st = capi.State(n)
    st.set_option(capi.SQ_OPT_JIT, jit)
    st.init_basis(5)
    st.flush()
    st.flush()
    psi = st.to_host()
    want = np.zeros(1 << n, dtype=np.complex128)
    want[5] = 1.0
    assert np.array_equal(psi, want)
    ops = circuits.random_all_gates(n, 40, seed=3)
    st.apply_ops(ops)
    st.flush()
    st.flush()
    assert np.abs(st.to_host() - oracle.run_ops(ops, n, state=want)).max() <= TOL
    st.close()


@pytest.mark.parametrize("jit", [0, 1])
def test_only_diagonal_and_phase_gates(jit):
    n = 12
    rng = np.random.default_rng(4)
    ops = [("Hadamard", (q,), ()) for q in range(n)]
    for _ in range(80):
        kind = rng.integers(5)
        q = tuple(int(x) for x in rng.choice(n, 2, replace=False))
        a = (float(rng.uniform(0, 6.28)),)
        ops.append([("RotZ", q[:1], a), ("ZZ", q, a), ("CPhaseShift", q, a), ("GPhase", (), a),
                    ("PhaseShift", q[:1], a)][kind])
    assert np.abs(run(ops, n, jit=jit) - oracle.run_ops(ops, n)).max() <= TOL


def test_global_phase_only():
    n = 7
    ops = [("Hadamard", (0,), ()), ("GPhase", (), (0.7,)), ("GPhase", (), (-2.1,))]
    assert np.abs(run(ops, n) - oracle.run_ops(ops, n)).max() <= TOL


@pytest.mark.parametrize("jit", [0, 1])
def test_every_qubit_targeted_and_extreme_controls(jit):
    n = 22
    ops = [("Hadamard", (q,), ()) for q in range(n)]
    ops += [("RotY", (q,), (0.1 * (q + 1),)) for q in range(n)]
    ops += [("CX", (0, n - 1), ()), ("CX", (n - 1, 0), ()), ("CCNot", (0, n - 1, n // 2), ()),
            ("CSwap", (n - 1, 0, 1), ()), ("Swap", (0, n - 1), ()), ("XX", (0, n - 1), (0.4,))]
    a = run(ops, n, jit=jit)
    assert np.abs(a - oracle.run_ops(ops, n)).max() <= TOL
    assert abs(np.vdot(a, a).real - 1.0) <= 1e-12
    # The same pattern at 14 qubits against the oracle.
    m = 14
    small = [op for op in circuits.random_all_gates(m, 0, seed=1)]
    small += [("Hadamard", (q,), ()) for q in range(m)]
    small += [("CX", (0, m - 1), ()), ("CCNot", (0, m - 1, m // 2), ()), ("CSwap", (m - 1, 0, 1), ())]
    assert np.abs(run(small, m, jit=jit) - oracle.run_ops(small, m)).max() <= TOL


def test_ragged_batches():
    # One circuit; circuits of the smallest batched size (4 qubits); mixed sizes.
    for sizes in ([9], [4, 4, 4], [4, 15, 5, 13, 4, 12]):
        b = capi.Batch(capi.SQ_C128)
        cases = []
        for i, n in enumerate(sizes):
            terms = circuits.random_pauli_hamiltonian(n, 6, seed=i + n)
            ops = circuits.random_all_gates(n, 30, seed=50 + i)
            cases.append((b.add_circuit(n, ops, b.add_hamiltonian(n, terms)), n, ops, terms))
        e = b.run()
        for cid, n, ops, terms in cases:
            want = oracle.expectation(oracle.run_ops(ops, n), n, terms)
            assert abs(e[cid] - want) <= 1e-11, (sizes, n)
        b.close()


def test_empty_batch_runs():
    b = capi.Batch(capi.SQ_C128)
    assert b.run().size == 0
    b.close()
