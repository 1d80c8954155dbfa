"""Structure groups of a batch energy run: streamed circuits that differ only
in their angles run as one multi-state JIT launch per sweep over all of
their states (sq_jit_msweep).  Energies and final states against the oracle,
and against the same batch with the groups turned off (SQ_BATCH_MULTI=0:
one CTA per circuit in batch_kernel)."""
import os

import numpy as np
import pytest

import oracle
from snuqs_b200 import capi, circuits

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _gpu(cuda_required):
    yield


def build(dtype, seed, counts):
    """counts: {n: number of VQE-ansatz circuits of n qubits}, plus one
    random all-gates circuit of 13 qubits (a structure of its own)."""
    rng = np.random.default_rng(seed)
    b = capi.Batch(dtype, keep_states=True)
    cases = []
    hams = {}
    for n, k in counts.items():
        terms = circuits.random_pauli_hamiltonian(n, 24, seed=n)
        hams[n] = (b.add_hamiltonian(n, terms), terms)
        for _ in range(k):
            th = rng.uniform(0, 2 * np.pi, 12 * n)
            ops = circuits.vqe_ansatz(n, th)
            cases.append((b.add_circuit(n, ops, hams[n][0]), n, ops, terms))
    terms = circuits.random_pauli_hamiltonian(13, 24, seed=99)
    hid = b.add_hamiltonian(13, terms)
    ops = circuits.random_all_gates(13, 120, seed=seed)
    cases.append((b.add_circuit(13, ops, hid), 13, ops, terms))
    return b, cases


def run_with(b, multi: bool):
    old = os.environ.get("SQ_BATCH_MULTI")
    os.environ["SQ_BATCH_MULTI"] = "1" if multi else "0"
    try:
        b.set_option(capi.SQ_BOPT_KEEP_STATES, 1)  # new plan version: replanned under the switch
        return b.run()
    finally:
        if old is None:
            del os.environ["SQ_BATCH_MULTI"]
        else:
            os.environ["SQ_BATCH_MULTI"] = old


@pytest.mark.parametrize("dtype,tol,stol", [(capi.SQ_C128, 1e-11, 1e-12), (capi.SQ_C64, 2e-5, 1e-5)])
def test_groups_against_oracle(dtype, tol, stol):
    # complex128 tiles are 2^11, complex64 2^12: a group needs >= 2 tiles per SM.
    k15 = 24 if dtype == capi.SQ_C128 else 40
    b, cases = build(dtype, seed=3, counts={20: 2, 15: k15, 9: 5})
    e = run_with(b, True)
    groups, grouped = b.groups()
    assert groups == 2 and grouped == 2 + k15
    checked = [c for c in cases if c[1] != 15] + [c for c in cases if c[1] == 15][:4]
    for cid, n, ops, terms in checked:
        ref = oracle.run_ops(ops, n)
        want = oracle.expectation(ref, n, terms)
        assert abs(e[cid] - want) <= tol * max(1.0, abs(want)), (cid, n)
        assert np.abs(b.state(cid) - ref).max() <= stol, (cid, n)
    b.close()


def test_groups_off_gives_the_same_energies():
    b, cases = build(capi.SQ_C128, seed=4, counts={16: 20, 12: 160, 10: 3})
    e_on = run_with(b, True)
    assert b.groups()[0] == 2
    e_off = run_with(b, False)
    assert b.groups() == (0, 0)
    assert np.abs(e_on - e_off).max() <= 1e-12
    b.close()


def test_groups_rerun_with_new_angles():
    """New angles for every circuit: same structures (no new kernels), new
    coefficients in the plan buffer, energies of the new angles."""
    rng = np.random.default_rng(8)
    b, cases = build(capi.SQ_C128, seed=5, counts={18: 4})
    run_with(b, True)
    new = []
    for cid, n, ops, terms in cases:
        if n != 18:
            continue
        th = rng.uniform(0, 2 * np.pi, 12 * n)
        b.set_angles(cid, th)
        new.append((cid, n, circuits.vqe_ansatz(n, th), terms))
    e = b.run()
    assert b.groups() == (1, 4)
    for cid, n, ops, terms in new:
        want = oracle.expectation(oracle.run_ops(ops, n), n, terms)
        assert abs(e[cid] - want) <= 1e-11 * max(1.0, abs(want))
    b.close()
