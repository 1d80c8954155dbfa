"""Regenerates the golden fixtures in this folder from the REFERENCE's own
CPU gate path (oracle/_ref/libsnuqs_ref.so, compiled from the reference
sources by oracle/Makefile).  Run from the repository root:

    python tests/golden/make_golden.py

Fixtures (all small):
  gate_matrices.npz   every reference gate's matrix at fixed angles
                      (gate_operations.cc constructors)
  per_gate.npz        a seeded 5-qubit state after each reference gate on
                      every ordered target tuple (cpu::applyGate)
  circuits.json +     op lists of seeded circuits and the reference's final
  circuits.npz        states: GHZ-12, the reference test's 33-gate random
                      mix (8 qubits, 200 gates), the 14-gate workload mix
                      (10 qubits, 120 gates), QV-6 with Unitary gates
"""
import itertools
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
import oracle  # noqa: E402
from snuqs_b200 import circuits  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
ANGLES = (0.7853981633974483 * 1.3, 2.1, -0.4)


def main():
    mats = {}
    for name in oracle.REFERENCE_GATES:
        na = oracle.gate_num_angles(name)
        mats[name] = oracle.ref_gate_matrix(name, ANGLES[:na])
    np.savez_compressed(os.path.join(HERE, "gate_matrices.npz"), angles=np.array(ANGLES), **mats)

    rng = np.random.default_rng(20241203)
    nq = 5
    psi0 = rng.standard_normal(1 << nq) + 1j * rng.standard_normal(1 << nq)
    psi0 /= np.linalg.norm(psi0)
    per = {"psi0": psi0}
    for name in oracle.REFERENCE_GATES:
        k = oracle.gate_qubits(name)
        na = oracle.gate_num_angles(name)
        for t in itertools.permutations(range(nq), k):
            s = psi0.copy()
            oracle.ref_apply_gate(s, nq, name, list(t), ANGLES[:na])
            per[f"{name}|{','.join(map(str, t))}"] = s
    np.savez_compressed(os.path.join(HERE, "per_gate.npz"), **per)

    cases = {
        "ghz12": (12, circuits.ghz(12)),
        "ref_mix_8q": (8, circuits.random_all_gates(8, 200, seed=7)),
        "workload_mix_10q": (10, circuits.random_mix(10, 120, seed=11)),
        "qv6": (6, circuits.quantum_volume(6, 6, seed=5)),
    }
    meta, states = {}, {}
    for key, (n, ops) in cases.items():
        states[key] = oracle.run_ops(ops, n, use_ref=True)
        meta[key] = {"n": n, "ops": [
            [op[0], list(op[1]), list(op[2])] + ([np.asarray(op[3]).real.tolist(),
                                                   np.asarray(op[3]).imag.tolist()]
                                                  if op[0] == "Unitary" else [])
            for op in ops]}
    with open(os.path.join(HERE, "circuits.json"), "w") as f:
        json.dump(meta, f)
    np.savez_compressed(os.path.join(HERE, "circuits.npz"), **states)
    print("wrote fixtures to", HERE)


if __name__ == "__main__":
    main()
