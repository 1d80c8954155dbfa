"""Batched circuits across GPUs: one process per GPU, each runs one batch
launch on its share of the circuits, and the per-circuit results are
gathered (torch.distributed: NCCL between GPUs, gloo on CPU).

Circuits are independent units, so there is no collective on the data path:
only the final per-circuit scalars (a few KB) cross between ranks.  Shares
are balanced by work (2^n amplitudes per circuit, longest-processing-time
first), not by count.
"""
from __future__ import annotations

import heapq
from typing import Callable, Sequence

import numpy as np


def partition(sizes: Sequence[int], world: int) -> list[list[int]]:
    """Circuit indices per rank: each circuit (largest 2^n first) goes to the
    rank with the least work so far; ties go to the lowest rank.  Every index
    appears exactly once; each rank's list is in ascending order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    heap = [(0, r) for r in range(world)]
    shares: list[list[int]] = [[] for _ in range(world)]
    order = sorted(range(len(sizes)), key=lambda i: (-(1 << int(sizes[i])), i))
    for i in order:
        load, r = heapq.heappop(heap)
        shares[r].append(i)
        heapq.heappush(heap, (load + (1 << int(sizes[i])), r))
    return [sorted(s) for s in shares]


def gather_results(local: np.ndarray, share: Sequence[int], total: int, rank: int, world: int,
                   group=None) -> np.ndarray:
    """Assembles per-circuit rows computed by every rank into one array in
    circuit order (all ranks receive it).  `local` has one row per index of
    this rank's `share` (a 1-D array is one value per circuit)."""
    import torch
    import torch.distributed as dist

    local = np.asarray(local, dtype=np.float64)
    row = local.shape[1:] if local.ndim > 1 else ()
    if world == 1:
        out = np.zeros((total,) + row)
        out[np.asarray(share, dtype=np.int64)] = local
        return out
    backend = dist.get_backend(group)
    device = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    # Pad every rank's rows to the largest share (all_gather needs equal sizes).
    counts = torch.tensor([len(share)], dtype=torch.int64, device=device)
    all_counts = [torch.zeros_like(counts) for _ in range(world)]
    dist.all_gather(all_counts, counts, group=group)
    cap = int(max(int(c.item()) for c in all_counts))
    width = int(np.prod(row)) if row else 1
    buf = torch.zeros((cap, 1 + width), dtype=torch.float64, device=device)
    if len(share):
        buf[: len(share), 0] = torch.as_tensor(np.asarray(share, dtype=np.float64), device=device)
        buf[: len(share), 1:] = torch.as_tensor(local.reshape(len(share), width), device=device)
    bufs = [torch.zeros_like(buf) for _ in range(world)]
    dist.all_gather(bufs, buf, group=group)
    out = np.zeros((total, width))
    for r in range(world):
        b = bufs[r].cpu().numpy()
        n = int(all_counts[r].item())
        out[b[:n, 0].astype(np.int64)] = b[:n, 1:]
    return out.reshape((total,) + row)


def run_sharded(sizes: Sequence[int], runner: Callable[[list[int]], np.ndarray], rank: int, world: int,
                group=None) -> np.ndarray:
    """Runs `runner(share)` (this rank's circuit indices -> one row per
    circuit, e.g. a batch launch's energies or gradients) on the partition
    share of `rank` and gathers the rows of every rank in circuit order."""
    share = partition(sizes, world)[rank]
    local = runner(share) if share else np.zeros((0,))
    return gather_results(local, share, len(sizes), rank, world, group)


def batch_runner(dtype: int, circuits_of: Callable[[int], tuple], n_params: int | None = None):
    """runner for run_sharded: builds one sq_batch from circuits_of(i) ->
    (n, ops, terms) for the share, runs it in one launch and returns the
    energies (n_params None) or [energy, gradient...] rows."""
    from . import capi

    def run(share: list[int]) -> np.ndarray:
        b = capi.Batch(dtype)
        hams = {}
        for i in share:
            n, ops, terms = circuits_of(i)
            key = (n, tuple((w, p) for w, p in terms))
            if key not in hams:
                hams[key] = b.add_hamiltonian(n, terms)
            b.add_circuit(n, ops, hams[key])
        try:
            if n_params is None:
                return b.run()
            e, g = b.run_gradients(n_params)
            return np.concatenate([e[:, None], g], axis=1)
        finally:
            b.close()

    return run
