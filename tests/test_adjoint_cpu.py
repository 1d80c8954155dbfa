"""Adjoint gradient, host logic: the reverse op list (adjoint_plan.cc) and the
two-state sweep plan, executed by the test-only emulator, against central
finite differences of the oracle's energy."""
import numpy as np
import pytest

import oracle
from snuqs_b200 import circuits
from tests.native import emulator

PARAM_GATES = ["RotX", "RotY", "RotZ", "PhaseShift", "CPhaseShift", "CPhaseShift00",
               "CPhaseShift01", "CPhaseShift10", "PSwap", "XY", "XX", "YY", "ZZ", "U", "PRx",
               "GPhase"]


def energy(n, ops, theta, terms):
    concrete = []
    for op in ops:
        if op[0] == "Unitary" or len(op) < 4:
            concrete.append(op[:3] if op[0] != "Unitary" else op)
            continue
        a = list(op[2])
        for j, p in enumerate(op[3]):
            if p >= 0:
                a[j] = theta[p] * (op[4][j] if len(op) > 4 else 1.0)
        concrete.append((op[0], op[1], tuple(a)))
    psi = oracle.run_ops(concrete, n)
    return oracle.expectation(psi, n, terms)


def bind(ops, theta):
    out = []
    for op in ops:
        if op[0] == "Unitary" or len(op) < 4:
            out.append(op)
            continue
        a = list(op[2])
        for j, p in enumerate(op[3]):
            if p >= 0:
                a[j] = theta[p] * (op[4][j] if len(op) > 4 else 1.0)
        out.append((op[0], op[1], tuple(a)) + tuple(op[3:]))
    return out


def fd_grad(n, ops, theta, terms, h=1e-5):
    g = np.zeros(len(theta))
    for p in range(len(theta)):
        tp, tm = theta.copy(), theta.copy()
        tp[p] += h
        tm[p] -= h
        g[p] = (energy(n, ops, tp, terms) - energy(n, ops, tm, terms)) / (2 * h)
    return g


def random_param_circuit(n, ngates, nparams, seed):
    rng = np.random.default_rng(seed)
    ops = [("Hadamard", (q,), ()) for q in range(n)]
    fixed = ["CX", "CZ", "Swap", "CCNot", "Hadamard", "ISwap", "CSwap"]
    for _ in range(ngates):
        if rng.random() < 0.7:
            name = PARAM_GATES[int(rng.integers(len(PARAM_GATES)))]
            k, na = circuits.GATES[name]
            q = tuple(int(x) for x in rng.choice(n, size=k, replace=False)) if k else ()
            params = tuple(int(rng.integers(nparams)) for _ in range(na))
            scales = tuple(float(rng.choice([1.0, -0.5, 2.0])) for _ in range(na))
            ops.append((name, q, (0.0,) * na, params, scales))
        else:
            name = fixed[int(rng.integers(len(fixed)))]
            k, _ = circuits.GATES[name]
            ops.append((name, tuple(int(x) for x in rng.choice(n, size=k, replace=False)), ()))
    return ops


@pytest.mark.parametrize("select,tile_bits", [(0, 10), (0, 7), (1, 7)])
@pytest.mark.parametrize("n,seed", [(5, 0), (8, 1), (11, 2), (13, 3)])
def test_adjoint_plan_matches_finite_differences(n, seed, select, tile_bits):
    nparams = 6
    ops = random_param_circuit(n, 40, nparams, seed)
    theta = np.random.default_rng(seed + 100).uniform(-3, 3, nparams)
    terms = circuits.random_pauli_hamiltonian(n, 12, seed=seed)
    e, g, sweeps = emulator.adjoint(n, bind(ops, theta), terms, nparams, tile_bits=tile_bits, select=select)
    assert abs(e - energy(n, ops, theta, terms)) < 1e-12
    assert np.abs(g - fd_grad(n, ops, theta, terms)).max() < 1e-8


def test_qaoa_adjoint_small():
    n, p = 8, 2
    edges = circuits.random_regular_graph(n, 3, seed=4)
    rng = np.random.default_rng(4)
    gam, bet = rng.uniform(0, np.pi, p), rng.uniform(0, np.pi, p)
    ops = [("Hadamard", (q,), ()) for q in range(n)]
    for l in range(p):
        ops += [("ZZ", (i, j), (gam[l],), (l,)) for i, j in edges]
        ops += [("RotX", (q,), (bet[l],), (p + l,)) for q in range(n)]
    theta = np.concatenate([gam, bet])
    terms = circuits.maxcut_hamiltonian(n, edges)
    e, g, _ = emulator.adjoint(n, ops, terms, 2 * p)
    assert abs(e - energy(n, ops, theta, terms)) < 1e-12
    assert np.abs(g - fd_grad(n, ops, theta, terms)).max() < 1e-8
