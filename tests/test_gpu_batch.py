"""Batched circuits in one persistent launch (sq_batch_*): energies and final
states of many uneven circuits against the oracle."""
import numpy as np
import pytest

import oracle
from snuqs_b200 import capi, circuits

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _gpu(cuda_required):
    yield


def make_batch(dtype, sizes, seed, keep=True, gates=80):
    rng = np.random.default_rng(seed)
    b = capi.Batch(dtype, keep_states=keep)
    hams, cases = {}, []
    for i, n in enumerate(sizes):
        if n not in hams:
            terms = circuits.random_pauli_hamiltonian(n, 24, seed=int(n))
            hams[n] = (b.add_hamiltonian(n, terms), terms)
        ops = circuits.random_all_gates(n, gates, seed=int(rng.integers(1 << 30)))
        cid = b.add_circuit(n, ops, hams[n][0])
        cases.append((cid, n, ops, hams[n][1]))
    return b, cases


@pytest.mark.parametrize("dtype,tol", [(capi.SQ_C128, 1e-11), (capi.SQ_C64, 2e-5)])
def test_batch_energies_and_states(dtype, tol):
    sizes = [4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 9, 11, 12, 4, 15]
    b, cases = make_batch(dtype, sizes, seed=1)
    e = b.run()
    for cid, n, ops, terms in cases:
        ref = oracle.run_ops(ops, n)
        want = oracle.expectation(ref, n, terms)
        assert abs(e[cid] - want) <= tol * max(1.0, abs(want)), (cid, n)
        assert np.abs(b.state(cid) - ref).max() <= (1e-12 if dtype == capi.SQ_C128 else 1e-5), n
    b.close()


def test_batch_vqe_rerun_with_new_angles():
    rng = np.random.default_rng(5)
    b = capi.Batch(capi.SQ_C128)
    cases = []
    for n in [8, 10, 12, 14, 16, 9, 13]:
        terms = circuits.random_pauli_hamiltonian(n, 32, seed=n)
        hid = b.add_hamiltonian(n, terms)
        th = rng.uniform(0, 2 * np.pi, 2 * n * 6)
        ops = circuits.vqe_ansatz(n, th)
        cases.append((b.add_circuit(n, ops, hid), n, terms))
    e1 = b.run()
    # New angles, same gates: the captured graph is replayed.
    for cid, n, terms in cases:
        th = rng.uniform(0, 2 * np.pi, 2 * n * 6)
        b.set_angles(cid, th)
        cases[cid] = (cid, n, terms, th)
    e2 = b.run()
    for cid, n, terms, th in cases:
        want = oracle.expectation(oracle.run_ops(circuits.vqe_ansatz(n, th), n), n, terms)
        assert abs(e2[cid] - want) <= 1e-11 * max(1.0, abs(want))
    assert not np.allclose(e1, e2)
    ms, ctas = b.last_timing()
    assert ms > 0 and ctas >= 1
    b.close()


def test_batch_rejects_mismatched_hamiltonian():
    b = capi.Batch()
    hid = b.add_hamiltonian(6, [(1.0, "ZZZZZZ")])
    with pytest.raises(capi.SqError):
        b.add_circuit(7, [("Hadamard", (0,), ())], hid)
    b.close()
