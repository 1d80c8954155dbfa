"""Noise channels on the device: density-matrix simulation (snuqs_b200.
density_matrix) against the oracle's column-by-column K rho K^H."""
import numpy as np
import pytest

import oracle
from snuqs_b200 import capi, circuits
from snuqs_b200 import noise_operations as no
from snuqs_b200.density_matrix import DensityMatrixSimulation

pytestmark = pytest.mark.gpu


def _channels(rng, n):
    q = lambda k: [int(x) for x in rng.choice(n, size=k, replace=False)]  # noqa: E731
    u = circuits.haar_unitary(2, rng)
    v = circuits.haar_unitary(2, rng)
    return [no.BitFlip(q(1), 0.1), no.PhaseFlip(q(1), 0.2), no.PauliChannel(q(1), 0.05, 0.1, 0.15),
            no.Depolarizing(q(1), 0.3), no.TwoQubitDepolarizing(q(2), 0.2),
            no.TwoQubitDephasing(q(2), 0.25), no.TwoQubitPauliChannel(q(2), {"XY": 0.1, "ZZ": 0.05}),
            no.AmplitudeDamping(q(1), 0.3), no.GeneralizedAmplitudeDamping(q(1), 0.2, 0.4),
            no.PhaseDamping(q(1), 0.35), no.Kraus(q(1), [np.sqrt(0.7) * u, np.sqrt(0.3) * v])]


@pytest.mark.parametrize("precision,tol", [("complex128", 1e-12), ("complex64", 2e-6)])
def test_noisy_circuit_against_oracle(cuda_required, precision, tol):
    n = 5
    rng = np.random.default_rng(9)
    gates = circuits.random_all_gates(n, 40, seed=9)
    chans = _channels(rng, n)
    sim = DensityMatrixSimulation(n, precision=precision)
    steps, ops = [], []
    for i, g in enumerate(gates):
        ops.append(g)
        steps.append(("unitary", circuits.op_matrix(g, oracle.gate_matrix), list(g[1])))
        if i % 4 == 3:
            ch = chans[(i // 4) % len(chans)]
            ops.append(ch)
            steps.append(("kraus", ch.matrices, list(ch.targets)))
    sim.evolve(ops)
    rho = oracle.density_evolve(n, steps)
    got = sim.density_matrix
    assert np.abs(got - rho).max() <= tol
    assert abs(sim.trace() - 1.0) <= tol
    assert np.abs(sim.probabilities - np.real(np.diag(rho))).max() <= tol
    terms = circuits.random_pauli_hamiltonian(n, 10, seed=3) + [(0.5, "ZZZZZ"), (0.2, "XYIZI")]
    from snuqs_b200.observables import matrix_of_terms

    want = float(np.real(np.trace(matrix_of_terms(terms) @ rho)))
    assert abs(sim.expectation(terms) - want) <= 10 * tol
    sim.close()


def test_pure_circuit_density_matrix_is_the_outer_product(cuda_required):
    n = 6
    ops = circuits.random_mix(n, 60, seed=2)
    psi = oracle.run_ops(ops, n)
    sim = DensityMatrixSimulation(n)
    sim.evolve(ops)
    assert np.abs(sim.density_matrix - np.outer(psi, psi.conj())).max() <= 1e-12
    sim.close()
