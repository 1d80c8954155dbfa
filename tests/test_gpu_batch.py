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


@pytest.mark.parametrize("dtype,tol", [(capi.SQ_C128, 1e-11), (capi.SQ_C64, 2e-5)])
def test_batch_launch_configurations_agree(dtype, tol):
    sizes = [5, 9, 10, 11, 12, 13, 14, 8]
    b, cases = make_batch(dtype, sizes, seed=21, keep=False, gates=60)
    want = {cid: oracle.expectation(oracle.run_ops(ops, n), n, terms) for cid, n, ops, terms in cases}
    for cfg in ({"tile_bits": 10, "low_bits": 3, "max_ops": 8, "ctas_per_sm": 1},
                {"tile_bits": 11, "low_bits": 0, "max_ops": 64, "ctas_per_sm": 0},
                {"tile_bits": 12, "low_bits": 3, "max_ops": 32, "ctas_per_sm": 2}):
        b.configure(cfg)
        e = b.run()
        for cid, w in want.items():
            assert abs(e[cid] - w) <= tol * max(1.0, abs(w)), (cfg, cid)
    b.close()


def test_batch_autotune_picks_a_candidate_and_keeps_results(tmp_path):
    b, cases = make_batch(capi.SQ_C128, [6, 10, 12, 13, 9, 11], seed=22, keep=False, gates=40)
    e0 = b.run()
    cache = str(tmp_path / "tune.json")
    cfg = b.autotune(reps=1, cache=cache)
    assert cfg["tile_bits"] in (10, 11, 12) and cfg["low_bits"] in (0, 3)
    assert cfg["max_ops"] in (32, 64) and 1 <= cfg["ctas_per_sm"] <= 4 and not cfg["cached"]
    e1 = b.run()
    assert np.abs(e1 - e0).max() <= 1e-11
    assert b.autotune(cache=cache)["cached"]
    b.close()


def test_batch_option_validation():
    b = capi.Batch(capi.SQ_C128)
    with pytest.raises(capi.SqError):
        b.set_option(capi.SQ_BOPT_TILE_BITS, 9)
    with pytest.raises(capi.SqError):
        b.set_option(capi.SQ_BOPT_MAX_OPS, 65)
    b.close()


def test_sharded_runner_on_one_rank_matches_batch():
    from snuqs_b200 import sharding

    sizes = [6, 9, 12, 13, 8]
    cs = {}
    for i, n in enumerate(sizes):
        cs[i] = (n, circuits.random_all_gates(n, 40, seed=300 + i), circuits.random_pauli_hamiltonian(n, 8, seed=i))
    got = sharding.run_sharded(sizes, sharding.batch_runner(capi.SQ_C128, lambda i: cs[i]), 0, 1)
    for i, (n, ops, terms) in cs.items():
        want = oracle.expectation(oracle.run_ops(ops, n), n, terms)
        assert abs(got[i] - want) <= 1e-11


def test_bench_sharded_batch_metric_one_rank():
    import bench

    out = bench.batch_metric_sharded("complex128", 0, 1, ncirc=64)
    assert out["circuits"] == 64 and out["energies_per_s"] > 0
    sizes, circuit_of = bench.vqe_batch_circuits(64)
    b = capi.Batch(capi.SQ_C128)
    for i in range(64):
        n, ops, terms = circuit_of(i)
        b.add_circuit(n, ops, b.add_hamiltonian(n, terms))
    assert abs(float(np.sum(b.run())) - out["energy_checksum"]) <= 1e-9
    b.close()
