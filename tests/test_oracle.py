"""The oracle is pinned before it is trusted: the C restatement must equal the
reference's own CPU path (oracle/_ref, compiled from the reference sources)
bit for bit, and both must reproduce the committed golden fixtures."""
import itertools
import os

import numpy as np
import pytest

import oracle
from tests.conftest import GOLDEN

ANGLE_SETS = [(0.3, 1.1, -2.0), (np.pi, np.pi / 2, 0.0), (5.9, 0.01, 3.3)]


@pytest.mark.parametrize("name", oracle.REFERENCE_GATES)
def test_restated_matrix_equals_reference_constructor(name):
    na = oracle.gate_num_angles(name)
    for a in ANGLE_SETS:
        assert np.array_equal(oracle.gate_matrix(name, a[:na]), oracle.ref_gate_matrix(name, a[:na]))


@pytest.mark.parametrize("name", oracle.REFERENCE_GATES)
def test_restated_apply_equals_reference_apply(name):
    rng = np.random.default_rng(3)
    nq = 5
    k, na = oracle.gate_qubits(name), oracle.gate_num_angles(name)
    for t in itertools.permutations(range(nq), k):
        psi = rng.standard_normal(1 << nq) + 1j * rng.standard_normal(1 << nq)
        a, b = psi.copy(), psi.copy()
        ang = ANGLE_SETS[0][:na]
        oracle.apply_matrix(a, nq, oracle.gate_matrix(name, ang), list(t))
        oracle.ref_apply_gate(b, nq, name, list(t), ang)
        assert np.array_equal(a, b), (name, t)


def test_golden_gate_matrices():
    g = np.load(os.path.join(GOLDEN, "gate_matrices.npz"))
    angles = g["angles"]
    for name in oracle.REFERENCE_GATES:
        na = oracle.gate_num_angles(name)
        assert np.array_equal(oracle.gate_matrix(name, angles[:na]), g[name]), name


def test_golden_per_gate_states():
    g = np.load(os.path.join(GOLDEN, "per_gate.npz"))
    ang = np.load(os.path.join(GOLDEN, "gate_matrices.npz"))["angles"]
    psi0 = g["psi0"]
    for key in g.files:
        if key == "psi0":
            continue
        name, t = key.split("|")
        targets = [int(x) for x in t.split(",")] if t else []
        s = psi0.copy()
        oracle.apply_matrix(s, 5, oracle.gate_matrix(name, ang[:oracle.gate_num_angles(name)]), targets)
        assert np.array_equal(s, g[key]), key


def test_golden_circuits(golden_circuits):
    for key, (n, ops, ref) in golden_circuits.items():
        assert np.array_equal(oracle.run_ops(ops, n), ref), key
        assert np.array_equal(oracle.run_ops(ops, n, use_ref=True), ref), key


def test_ghz_known_answer(golden_circuits):
    n, ops, ref = golden_circuits["ghz12"]
    want = np.zeros(1 << n, dtype=np.complex128)
    want[0] = want[-1] = np.sqrt(0.5)
    assert np.allclose(ref, want, atol=1e-15)


def test_pseudo_sort_matches_definition():
    # Descending by min target among gates on disjoint qubits; GPhase first;
    # gates sharing a qubit keep their order (transpile.py:33-89).
    tl = [(0,), (3,), (1, 2), (), (2,), (5, 4)]
    order = oracle.pseudo_sort_descending(tl)
    assert order[0] == 3  # the global phase moves to the front
    pos = {o: i for i, o in enumerate(order)}
    assert pos[2] < pos[4]  # (1,2) and (2,) share qubit 2
    assert sorted(order) == list(range(len(tl)))


def test_expectation_restatement():
    rng = np.random.default_rng(1)
    n = 4
    psi = rng.standard_normal(16) + 1j * rng.standard_normal(16)
    psi /= np.linalg.norm(psi)
    # dense check of the Pauli-string convention: character q acts on qubit q = index bit n-1-q
    P = {"I": np.eye(2), "X": np.array([[0, 1], [1, 0]]), "Y": np.array([[0, -1j], [1j, 0]]),
         "Z": np.diag([1, -1])}
    for s in ["XIYZ", "ZZII", "IYIY", "XXXX"]:
        m = P[s[0]]
        for ch in s[1:]:
            m = np.kron(m, P[ch])
        want = np.real(np.vdot(psi, m @ psi))
        assert abs(oracle.expectation(psi, n, [(1.0, s)]) - want) < 1e-14
