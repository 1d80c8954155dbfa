"""Host logic of the fused path, no GPU: the fusion planner and the gate
structure analysis, executed by the test-only plan emulator
(tests/native/plan_emulator.cc) with the kernels' index arithmetic, against
the oracle."""
import numpy as np
import pytest

import oracle
from snuqs_b200 import circuits
from tests.native import emulator


def gates_of(ops):
    return [(circuits.op_matrix(op, oracle.gate_matrix), op[1], [], []) for op in ops]


@pytest.mark.parametrize("n", [4, 5, 7, 9, 11, 12, 13, 15])
@pytest.mark.parametrize("reorder", [True, False, "select", "noselect"])
def test_plans_match_oracle_all_gates(n, reorder):
    for seed in range(2):
        ops = circuits.random_all_gates(n, 120, seed=seed)
        ref = oracle.run_ops(ops, n)
        for tb in (12, 9, 7):
            psi, sweeps, _ = emulator.run(oracle.basis_state(n), n, gates_of(ops), tb, reorder)
            assert np.abs(psi - ref).max() <= 1e-12, (n, seed, tb)


def test_plans_match_oracle_golden(golden_circuits):
    for key, (n, ops, ref) in golden_circuits.items():
        psi, _, _ = emulator.run(oracle.basis_state(n), n, gates_of(ops))
        assert np.abs(psi - ref).max() <= 1e-12, key


def test_fusion_packs_many_gates_per_sweep():
    ops = circuits.random_mix(20, 400, seed=1234)
    ref = oracle.run_ops(ops, 20)
    psi, sweeps, unfused = emulator.run(oracle.basis_state(20), 20, gates_of(ops))
    assert np.abs(psi - ref).max() <= 1e-12
    assert unfused == 0
    assert sweeps <= 40  # >= 10 gates per sweep


def test_controls_and_large_unitaries():
    rng = np.random.default_rng(9)
    n = 11
    gates = []
    for i in range(40):
        k = int(rng.integers(1, 6))  # up to 5 targets: k = 5 takes the unfused path
        qs = [int(x) for x in rng.choice(n, size=k + 2, replace=False)]
        u = circuits.haar_unitary(1 << k, rng)
        nc = int(rng.integers(0, 3))
        ctrl, vals = qs[k:k + nc], [int(v) for v in rng.integers(0, 2, size=nc)]
        gates.append((u, qs[:k], ctrl, vals))
    psi0 = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    ref = psi0.copy()
    for u, q, c, v in gates:
        # controlled(u) as a dense matrix over controls + targets
        kk = len(c) + len(q)
        D = 1 << kk
        full = np.eye(D, dtype=np.complex128)
        cidx = int("".join(map(str, v)), 2) if c else 0
        blk = cidx << len(q)
        full[blk:blk + (1 << len(q)), blk:blk + (1 << len(q))] = u
        oracle.apply_matrix(ref, n, full, list(c) + list(q))
    for reorder in (True, "select"):
        psi, sweeps, unfused = emulator.run(psi0, n, gates, 9, reorder)
        assert np.abs(psi - ref).max() <= 1e-12
        assert unfused > 0


def test_tile_selection_and_phase_scheduling_reduce_work():
    n = 24
    g = gates_of(circuits.random_mix(n, 400, seed=77))
    plain = emulator.plan_stats(n, g, tile_bits=11, reorder="noselect")
    sel = emulator.plan_stats(n, g, tile_bits=11, reorder="select")
    assert sel["ops"] == plain["ops"] == 400
    assert sel["sweeps"] < plain["sweeps"]
    assert sel["phases"] < 0.85 * plain["phases"]


@pytest.mark.parametrize("seed", range(3))
def test_selected_plans_match_oracle_on_larger_states(seed):
    n = 16
    ops = circuits.random_all_gates(n, 300, seed=40 + seed)
    ref = oracle.run_ops(ops, n)
    for tb in (7, 9, 11):
        psi, _, _ = emulator.run(oracle.basis_state(n), n, gates_of(ops), tb, "select")
        assert np.abs(psi - ref).max() <= 1e-12, tb


@pytest.mark.parametrize("low_bits", [1, 2, 3, 4, 6])
def test_low_bit_counts_match_oracle(low_bits):
    n = 15
    ops = circuits.random_all_gates(n, 200, seed=60 + low_bits)
    ref = oracle.run_ops(ops, n)
    for tb, ro in ((11, "select"), (10, True), (12, "noselect")):
        psi, _, _ = emulator.run(oracle.basis_state(n), n, gates_of(ops), tb, ro, low_bits)
        assert np.abs(psi - ref).max() <= 1e-12, (tb, ro)


def test_diagonal_and_identity_gates_fold():
    n = 10
    ops = [("Hadamard", (q,), ()) for q in range(n)]
    ops += [("RotZ", (q,), (0.1 * q,)) for q in range(n)]
    ops += [("ZZ", (q, (q + 3) % n), (0.3,)) for q in range(n)]
    ops += [("Identity", (2,), ()), ("GPhase", (), (0.25,)), ("CPhaseShift10", (1, 7), (1.0,))]
    ref = oracle.run_ops(ops, n)
    psi, sweeps, _ = emulator.run(oracle.basis_state(n), n, gates_of(ops))
    assert np.abs(psi - ref).max() <= 1e-12
    assert sweeps == 1


@pytest.mark.parametrize("n,tb,lb", [(14, 9, 3), (18, 11, 3), (20, 11, 5), (21, 10, 4), (22, 11, 3)])
def test_remapping_plans_match_oracle_and_save_sweeps(n, tb, lb):
    """Qubit remapping: sweeps store their tiles with low bits exchanged for
    the next sweep's hot bits; the plan still ends in the original order
    (the emulator stores through each sweep's output map)."""
    for ops in (circuits.random_mix(n, 300, seed=n), circuits.random_all_gates(n, 200, seed=n + 1),
                circuits.quantum_volume(n, 8, seed=n + 2)):
        ref = oracle.run_ops(ops, n)
        psi, sweeps, _ = emulator.run(oracle.basis_state(n), n, gates_of(ops), tb, "remap", lb)
        assert np.abs(psi - ref).max() <= 1e-12, n
        _, plain, _ = emulator.run(oracle.basis_state(n), n, gates_of(ops), tb, "select", lb)
        assert sweeps <= plain + 1


def test_remapping_saves_sweeps_on_the_benchmark_mix():
    g = gates_of(circuits.random_mix(30, 400, seed=1234))
    plain = emulator.plan_stats(30, g, tile_bits=11, reorder="select", low_bits=3)["sweeps"]
    remap = emulator.plan_stats(30, g, tile_bits=11, reorder="remap", low_bits=3)["sweeps"]
    assert remap < plain


def _param_circuit(n, angles):
    """Rotations (RotX/RotY/RotZ/PhaseShift/ZZ/XX/U), fixed CX/CZ/H and a
    controlled rotation, angles from `angles` in order."""
    it = iter(angles)
    ops = []
    for l in range(3):
        for q in range(n):
            ops.append(("RotY", (q,), (next(it),)))
            ops.append(("RotZ", (q,), (next(it),)))
        for q in range(0, n - 1, 2):
            ops.append(("ZZ", (q, q + 1), (next(it),)))
        for q in range(n - 1):
            ops.append(("CX", (q, q + 1), ()))
        ops.append(("XX", (0, n - 1), (next(it),)))
        ops.append(("PhaseShift", (n // 2,), (next(it),)))
        ops.append(("U", (1,), (next(it), next(it), next(it))))
        ops.append(("CPhaseShift", (2, n - 2), (next(it),)))
        ops.append(("Hadamard", (3,), ()))
    return ops


@pytest.mark.parametrize("n,tb,reorder", [(13, 9, "select"), (14, 10, True), (12, 8, "noselect"), (16, 11, "select")])
def test_rebuilt_plans_match_oracle(n, tb, reorder):
    """A plan made for one set of angles, re-emitted for another by
    rebuild_plan (same gates, no planning), gives the oracle's state for the
    new angles; an angle that turns a gate into the identity (dropped by the
    op analysis) changes the op signature and the plan is made anew."""
    rng = np.random.default_rng(n)
    na = len([a for op in _param_circuit(n, iter(lambda: 0.5, None)) for a in op[2]])
    a, b = rng.uniform(0.1, 3.0, na), rng.uniform(0.1, 3.0, na)
    ops_a, ops_b = _param_circuit(n, a), _param_circuit(n, b)
    ref = oracle.run_ops(ops_b, n)
    psi, sweeps, rebuilt = emulator.run_rebuilt(oracle.basis_state(n), n, gates_of(ops_a), gates_of(ops_b),
                                                tb, reorder)
    assert rebuilt and sweeps > 1
    assert np.abs(psi - ref).max() <= 1e-12
    c = b.copy()
    c[1] = 0.0  # RotZ(0) is the identity: dropped, so the ops differ
    ops_c = _param_circuit(n, c)
    psi, _, rebuilt = emulator.run_rebuilt(oracle.basis_state(n), n, gates_of(ops_a), gates_of(ops_c), tb, reorder)
    assert not rebuilt
    assert np.abs(psi - oracle.run_ops(ops_c, n)).max() <= 1e-12
