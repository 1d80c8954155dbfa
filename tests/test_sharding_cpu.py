"""Batches sharded across ranks (snuqs_b200.sharding), without a GPU: the
work partition, and the gather of per-circuit rows over a world-size-2 gloo
process group, with the oracle standing in for each rank's batch launch."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from snuqs_b200 import sharding


def test_partition_covers_every_circuit_once_and_balances_work():
    rng = np.random.default_rng(0)
    sizes = [int(x) for x in rng.integers(8, 21, size=4096)]
    for world in (1, 2, 3, 8):
        shares = sharding.partition(sizes, world)
        flat = sorted(i for s in shares for i in s)
        assert flat == list(range(len(sizes)))
        loads = [sum(1 << sizes[i] for i in s) for s in shares]
        assert max(loads) - min(loads) <= (1 << max(sizes))


def test_partition_more_ranks_than_circuits():
    shares = sharding.partition([10, 12], 4)
    assert sorted(i for s in shares for i in s) == [0, 1]
    assert sum(1 for s in shares if not s) == 2


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, sizes, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import oracle
        from snuqs_b200 import circuits

        def circuit_of(i):
            n = sizes[i]
            ops = circuits.random_all_gates(n, 30, seed=100 + i)
            return n, ops, circuits.random_pauli_hamiltonian(n, 6, seed=i)

        def runner(share):
            rows = []
            for i in share:
                n, ops, terms = circuit_of(i)
                e = oracle.expectation(oracle.run_ops(ops, n), n, terms)
                rows.append([e, float(rank), float(i)])
            return np.asarray(rows)

        out = sharding.run_sharded(sizes, runner, rank, world)
        q.put((rank, out))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_gather_over_two_gloo_ranks_matches_serial():
    import oracle
    from snuqs_b200 import circuits

    sizes = [4, 6, 5, 7, 4, 8, 6, 5, 4]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, sizes, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = dict(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    shares = sharding.partition(sizes, 2)
    for r in range(2):
        out = results[r]
        assert out.shape == (len(sizes), 3)
        for i, n in enumerate(sizes):
            ops = circuits.random_all_gates(n, 30, seed=100 + i)
            want = oracle.expectation(oracle.run_ops(ops, n), n, circuits.random_pauli_hamiltonian(n, 6, seed=i))
            assert abs(out[i, 0] - want) <= 1e-12
            assert out[i, 2] == i
            assert i in shares[int(out[i, 1])]
    assert np.array_equal(results[0], results[1])
