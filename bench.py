"""Benchmark: fused gate sweeps on a 30-qubit complex128 state (one B200).

Workload (one "step"): the seeded 400-gate random mix (RotX/RotY/RotZ/U/
PhaseShift, CX/CZ/Swap/ISwap/XX/YY/ZZ, CCNot/CSwap; seed 1234) applied to a
2^30-amplitude complex128 state resident in HBM (16 GiB, far above the 126 MB
L2, so no flush is needed between steps).

Metric: effective gate-sweep bandwidth = gates x 2 x 16 B x 2^n / step time,
the figure the reference's per-gate path is measured in (each reference gate
is one full read+write sweep).  The roofline object reports the real HBM
bandwidth of the fused sweep kernel: 2 x 16 B x 2^n per launch over its
CUDA-event-timed launch duration, against the measured copy bandwidth.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

--impl reference times the reference's own CPU gate path (cpu::applyGate
compiled from the reference sources into oracle/_ref) on the host cores,
one gate of the same circuit per step.  With N > 1 (torchrun), every rank runs
an independent replica (the single-state path does not shard), the step time
is the max over ranks, and the value is the sum over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_QUBITS = 30
N_GATES = 400
SEED = 1234
AMP_BYTES = 16
FALLBACK_HBM_GBS = 6650.0
# DRAM bytes (read + write) per amplitude of one JIT sweep launch, from one ncu
# capture of the same random-mix generator at 26 qubits complex128 (2.0917 GB
# per launch / 2^26 amplitudes; profiles/sq_jit_sweep_random_mix_26q_c128_ncu_full.md),
# scaled to the benchmark's 2^n amplitudes.
NCU_DRAM_BYTES_PER_AMP = {"complex128": 2.0917e9 / (1 << 26)}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--qubits", type=int, default=N_QUBITS)
    p.add_argument("--gates", type=int, default=N_GATES)
    p.add_argument("--precision", default="complex128", choices=["complex128", "complex64"])
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-adjoint", action="store_true")
    p.add_argument("--no-batch", action="store_true")
    p.add_argument("--no-configs", action="store_true",
                   help="skip the complex64 comparison and the other workload configurations")
    p.add_argument("--tile-bits", type=int, default=0, help="override the engine's tile size")
    p.add_argument("--low-bits", type=int, default=0,
                   help="override the contiguous low bits of every tile")
    p.add_argument("--adjoint-only", action="store_true",
                   help="only the QAOA-26 adjoint gradient, without the parameter-shift comparison "
                        "(a short command for profiling the adjoint kernels)")
    p.add_argument("--batch-only", action="store_true",
                   help="only the VQE energy batch, default configuration, no autotuning or oracle "
                        "check (a short command for profiling the batch kernels)")
    p.add_argument("--kernel-tour", action="store_true",
                   help="run each kernel family once on a small case (for ncu captures) "
                        "instead of the benchmark line")
    p.add_argument("--op-cost", action="store_true",
                   help="print the per-gate cost inside one fused sweep for each sweep-op kind "
                        "(--qubits, default 27) instead of the benchmark line")
    return p.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        except Exception:
            pass
        finally:
            try:
                os.unlink(self.path)
            except Exception:
                pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


def circuit(n, ngates):
    from snuqs_b200 import circuits
    return circuits.random_mix(n, ngates, seed=SEED)


# ---------------------------------------------------------------------------
# Reference CPU path (oracle/_ref: the reference's cpu::applyGate)
# ---------------------------------------------------------------------------
def host_ram_ok(n):
    try:
        import psutil

        return psutil.virtual_memory().available > 2.5 * (1 << n) * AMP_BYTES
    except Exception:
        return False


def pseudo_sorted(ops):
    """The circuit in the order the reference applies it: its
    pseudo_sort_operations_descending (transpile.py:74-89), restated in the
    oracle."""
    import oracle

    return [ops[i] for i in oracle.pseudo_sort_descending([op[1] for op in ops])]


def ref_apply(psi, n, op):
    import oracle

    if op[0] == "Unitary":
        oracle.ref_apply_matrix(psi, n, op[3], op[1])
    else:
        oracle.ref_apply_gate(psi, n, op[0], op[1], op[2])


def run_reference(args, rank, world):
    """The reference's own CPU gate path on the host cores: every gate of the
    circuit, in the reference's pseudo-sort order, one cpu::applyGate each.
    Warm-up steps apply one gate each; the timed steps together apply all
    gates once (ceil(gates / steps) per step)."""
    if rank != 0:
        return
    import oracle

    n, ops = args.qubits, pseudo_sorted(circuit(args.qubits, args.gates))
    if not host_ram_ok(n):
        print(json.dumps({"impl": "reference", "unavailable":
                          f"host RAM below 2.5x the {n}-qubit state for the reference CPU path"}))
        return
    psi = np.zeros(1 << n, dtype=np.complex128)
    oracle.ref_initialize_basis_z(psi, n)
    for w in range(args.warmup):
        ref_apply(psi, n, ops[w % len(ops)])
    per = -(-len(ops) // args.steps)
    t0 = time.perf_counter()
    done = 0
    for s in range(args.steps):
        for op in ops[s * per:(s + 1) * per]:
            ref_apply(psi, n, op)
            done += 1
    t = time.perf_counter() - t0
    value = done * 2 * AMP_BYTES * (1 << n) / t / 1e9
    threads = oracle.ref().ref_max_threads()
    sample = (f"all {done} gates of the {n}-qubit circuit in the reference's pseudo-sort order, "
              f"{per} per timed step, {t:.1f} s, OMP threads {threads}")
    print(json.dumps({
        "impl": "reference", "metric": metric_name(n, args.precision), "value": round(value, 3),
        "unit": "GB/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(t / args.steps * 1e3, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": f"synthetic: seeded random gate mix (seed {SEED})",
        "config": config(n, args), "cpu_baseline": {
            "value": round(value, 3), "unit": "GB/s", "cores": threads, "kind": "reference",
            "sample": sample},
        "e2e": {"value": round(value, 3), "unit": "GB/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0}}))


def metric_name(n, precision):
    return (f"{n}q {precision} random-mix effective gate-sweep GB/s "
            f"(gates x 2 x amp bytes x 2^n / step time)")


def config(n, args):
    return {"workload": f"random_mix_{n}q_{args.precision}_{args.gates}g", "qubits": n,
            "gates": args.gates, "precision": args.precision, "seed": SEED,
            "state_bytes": (1 << n) * (16 if args.precision == "complex128" else 8),
            "l2": "state far above the 126 MB L2; no flush between steps",
            "parallelism": "replicas"}


# ---------------------------------------------------------------------------
# Our engine
# ---------------------------------------------------------------------------
def op_cost(args):
    """Marginal cost of one gate inside a fused sweep, per sweep-op kind: a
    sweep of 1 and of 31 gates of one kind on the same 4 qubits (one register
    phase), CUDA-event timed over 5 repetitions each; the slope over 30 gates
    is the cost of one gate (an odd count, so that products of self-inverse
    gates do not cancel to the identity).  One JSON line per kind."""
    import torch

    from snuqs_b200 import capi, circuits

    n = args.qubits if args.qubits != N_QUBITS else 27
    dtype = capi.SQ_C128 if args.precision == "complex128" else capi.SQ_C64
    amp = 16 if dtype == capi.SQ_C128 else 8
    rng = np.random.default_rng(SEED)
    a, b, c, d = n - 8, n - 9, n - 10, n - 11  # four qubits on high index bits 7..10
    u2 = circuits.haar_unitary(4, rng)
    kinds = [
        ("PhaseShift", "conditional phase", lambda i: ("PhaseShift", ((a, b, c, d)[i % 4],), (0.3,))),
        ("RotZ", "diagonal", lambda i: ("RotZ", ((a, b, c, d)[i % 4],), (0.3,))),
        ("PauliX", "anti-diagonal, pure", lambda i: ("PauliX", ((a, b, c, d)[i % 4],), ())),
        ("PauliY", "anti-diagonal", lambda i: ("PauliY", ((a, b, c, d)[i % 4],), ())),
        ("RotX", "rotation form, imaginary", lambda i: ("RotX", ((a, b, c, d)[i % 4],), (0.3,))),
        ("RotY", "rotation form, real", lambda i: ("RotY", ((a, b, c, d)[i % 4],), (0.3,))),
        ("XX", "2-qubit rotation form", lambda i: ("XX", ((a, b), (c, d))[i % 2], (0.3,))),
        ("Swap", "middle swap, pure", lambda i: ("Swap", ((a, b), (c, d))[i % 2], ())),
        ("ISwap", "middle swap", lambda i: ("ISwap", ((a, b), (c, d))[i % 2], ())),
        ("U", "dense 1q", lambda i: ("U", ((a, b, c, d)[i % 4],), (0.1, 0.2, 0.3))),
        ("CX", "control in registers", lambda i: ("CX", ((a, b), (c, d))[i % 2], ())),
        ("CX", "control outside the tile", lambda i: ("CX", (0, (a, b, c, d)[i % 4]), ())),
        ("ZZ", "diagonal", lambda i: ("ZZ", ((a, b), (c, d))[i % 2], (0.3,))),
        ("Unitary", "dense 2q", lambda i: ("Unitary", ((a, b), (c, d))[i % 2], (), u2)),
    ]
    st = capi.State(n, dtype)
    st.init_basis(0)
    floor_ms = 2 * amp * (1 << n) / (measured_peak()[0] * 1e9) * 1e3
    for name, kind, mk in kinds:
        times = {}
        for count in (1, 31):
            ops = [mk(i) for i in range(count)]
            st.apply_ops(ops)  # warm-up (and JIT compile)
            st.flush()
            torch.cuda.synchronize()
            st.sweep_timing()
            st.set_option(capi.SQ_OPT_TIMING, 1)
            for _ in range(5):
                st.apply_ops(ops)
                st.flush()
            st.set_option(capi.SQ_OPT_TIMING, 0)
            ms, launches = st.sweep_timing()
            times[count] = (ms / max(1, launches), launches / 5)
        slope = (times[31][0] - times[1][0]) / 30
        print(json.dumps({"gate": name, "kind": kind, "qubits": n, "precision": args.precision,
                          "sweep_ms_1": round(times[1][0], 4), "sweep_ms_31": round(times[31][0], 4),
                          "sweeps_per_flush": times[31][1],
                          "ps_per_amp_per_gate": round(slope * 1e-3 / (1 << n) * 1e12, 4),
                          "hbm_floor_ms": round(floor_ms, 4)}))
    st.close()


def kernel_tour():
    """Each kernel family once, on cases sized for an ncu capture (states of
    2^22-2^24 amplitudes, above the 126 MB L2 where it matters): unfused gate
    kernel, Pauli expectation, single-circuit adjoint (Pauli apply, two-state
    sweeps, inner-product reduction), batched energies, batched gradients."""
    import torch

    from snuqs_b200 import adjoint, capi, circuits

    n = 24
    st = capi.State(n)
    st.set_option(capi.SQ_OPT_FUSION, 0)
    st.init_basis(0)
    st.apply_ops(circuits.random_mix(n, 8, seed=SEED))  # gate_kernel, one launch per gate
    st.flush()
    terms = circuits.random_pauli_hamiltonian(n, 16, seed=SEED)
    e = st.expectation(terms)  # pauli_expect_kernel
    st.close()
    ops, qterms, theta = qaoa_workload(22, 2)
    ws = adjoint.Workspace(22)
    e2, g = adjoint.adjoint_gradient(ws, ops, theta, qterms, 4)  # adjoint kernels
    ws.close()
    rng = np.random.default_rng(SEED)
    b = capi.Batch(capi.SQ_C128)
    hams = {k: b.add_hamiltonian(k, circuits.random_pauli_hamiltonian(k, 16, seed=k)) for k in range(8, 17)}
    for _ in range(256):
        k = int(rng.integers(8, 17))
        b.add_circuit(k, circuits.vqe_ansatz(k, rng.uniform(0, 2 * np.pi, 12 * k)), hams[k])
    eb = b.run()  # batch_kernel
    b.close()
    ops16, t16, _ = qaoa_workload(16, 4)
    b = capi.Batch(capi.SQ_C128)
    h16 = b.add_hamiltonian(16, t16)
    for th in rng.uniform(0, np.pi, (64, 8)):
        b.add_circuit(16, adjoint.bind(ops16, th), h16)
    eg, gg = b.run_gradients(8)  # batch_adjoint_kernel
    b.close()
    torch.cuda.synchronize()
    print(json.dumps({"kernel_tour": "ok", "expectation": e, "adjoint_energy": e2,
                      "batch_energy_0": float(eb[0]), "batch_grad_00": float(gg[0, 0])}))


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.kernel_tour:
        kernel_tour()
        return
    if args.adjoint_only:
        print(json.dumps(adjoint_metric(args.precision, shift=False)))
        return
    if args.batch_only:
        print(json.dumps(batch_metric(args.precision, tune=False)))
        return
    if args.op_cost:
        op_cost(args)
        return
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    _run_ours(args, rank, world, local)


def _run_ours(args, rank, world, local):
    import torch
    import torch.distributed as dist

    from snuqs_b200 import _C, capi, circuits

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    n = args.qubits
    amp = 16 if args.precision == "complex128" else 8
    dtype = capi.SQ_C128 if args.precision == "complex128" else capi.SQ_C64
    ops = circuit(n, args.gates)
    mats = [circuits.op_matrix(op, capi.gate_matrix) for op in ops]
    stream = torch.cuda.current_stream().cuda_stream

    st = capi.State(n, dtype, stream=stream)
    st.init_basis(0)
    if args.tile_bits:
        st.set_option(capi.SQ_OPT_TILE_BITS, args.tile_bits)
    if args.low_bits:
        st.set_option(capi.SQ_OPT_LOW_BITS, args.low_bits)

    def step():
        for op, m in zip(ops, mats):
            st.apply_matrix(m, op[1])
        st.flush()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    l0 = st.launches()
    st.set_option(capi.SQ_OPT_TIMING, 1)
    jit0 = capi.jit_info()[1]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record()
        for _ in range(args.steps):
            step()
        ev1.record()
        torch.cuda.synchronize()
    st.set_option(capi.SQ_OPT_TIMING, 0)
    ms = ev0.elapsed_time(ev1) / args.steps
    sweep_ms, sweeps = st.sweep_timing()
    launches = st.launches() - l0
    jit_sweeps = capi.jit_info()[1] - jit0
    if world > 1:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = world * args.gates * 2 * amp * (1 << n) / (ms * 1e-3) / 1e9
    sweeps_per_step = sweeps / args.steps
    per_launch_ms = sweep_ms / max(1, sweeps)
    alg_bytes = 2 * amp * (1 << n)
    peak, peak_kind = measured_peak()
    achieved = alg_bytes / (per_launch_ms * 1e-3) / 1e9
    clocks = clk.summary()

    out = {
        "metric": metric_name(n, args.precision), "value": round(value, 2), "unit": "GB/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if dtype == capi.SQ_C128 else "f32",
        "data": f"synthetic: seeded random gate mix (seed {SEED})", "config": config(n, args),
        "gate_sweeps_per_s": round(world * args.gates / (ms * 1e-3), 2),
        "fused_sweeps_per_step": sweeps_per_step,
        "gates_per_sweep": round(args.gates / max(1e-9, sweeps_per_step), 2),
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                     "unit": "GB/s", "frac": round(achieved / peak, 4),
                     "traffic": (round(NCU_DRAM_BYTES_PER_AMP[args.precision] * (1 << n))
                                 if args.precision in NCU_DRAM_BYTES_PER_AMP and jit_sweeps == sweeps
                                 else None),
                     "traffic_note": "ncu dram read+write bytes per launch at 26 qubits, scaled by 2^(n-26)",
                     "kernel": ("sq_jit_sweep (NVRTC-specialised sweep, " if jit_sweeps == sweeps
                                else "sq::sweep_kernel (") +
                               ("double)" if dtype == capi.SQ_C128 else "float)"),
                     "jit_sweeps": jit_sweeps,
                     "per_launch_ms": round(per_launch_ms, 4),
                     "algorithmic_bytes_per_launch": alg_bytes, "peak_source": peak_kind},
        "gpu_launches": launches, "clocks": clocks,
    }

    if world == 1 and rank == 0 and dtype == capi.SQ_C128 and not args.no_configs:
        try:
            out["complex64"] = complex64_metric(st, n, ops, mats, args)
        except Exception as e:
            out["complex64"] = {"note": f"complex64 run failed: {e}"}
    st.close()
    if world == 1 and rank == 0 and not args.no_configs:
        out["configs"] = config_metrics()
    if world == 1 and rank == 0 and not args.no_e2e:
        try:
            out["e2e"] = e2e(n, ops, args, amp)
        except Exception as e:  # report, do not lose the device-timed line
            out["e2e"] = {"value": None, "unit": "GB/s", "note": f"e2e failed: {e}"}
        if dtype == capi.SQ_C128 and not args.no_configs and out["e2e"].get("value"):
            try:
                out["e2e"]["complex64"] = e2e(n, ops, args, 8, precision="complex64")
            except Exception as e:
                out["e2e"]["complex64"] = {"note": f"complex64 e2e failed: {e}"}
    with_c64 = dtype == capi.SQ_C128 and not args.no_configs
    if world == 1 and rank == 0 and not args.no_adjoint:
        ref = {}
        try:
            out["adjoint"] = adjoint_metric(args.precision, keep=ref)
        except Exception as e:
            out["adjoint"] = {"note": f"adjoint failed: {e}"}
        if with_c64 and ref:
            try:
                got = {}
                a64 = adjoint_metric("complex64", shift=False, keep=got)
                a64 = {k: a64[k] for k in ("workload", "adjoint_ms", "forward_sweeps_ms", "reverse_sweeps_ms",
                                           "reverse_sweep_frac", "roofline")}
                a64["max_abs_gradient_error_vs_complex128"] = float(np.abs(got["gradient"] - ref["gradient"]).max())
                a64["energy_error_vs_complex128"] = abs(got["energy"] - ref["energy"])
                out["adjoint"]["complex64"] = a64
            except Exception as e:
                out["adjoint"]["complex64"] = {"note": f"complex64 adjoint failed: {e}"}
    if world == 1 and rank == 0 and not args.no_batch:
        ref = {}
        try:
            out["batch"] = batch_metric(args.precision, keep=ref)
        except Exception as e:
            out["batch"] = {"note": f"batch failed: {e}"}
        if with_c64 and ref:
            try:
                out["batch"]["complex64"] = batch_complex64_metric(ref["energies"])
            except Exception as e:
                out["batch"]["complex64"] = {"note": f"complex64 batch failed: {e}"}
        try:
            out["qaoa_batch"] = qaoa_batch_metric(args.precision)
        except Exception as e:
            out["qaoa_batch"] = {"note": f"qaoa batch failed: {e}"}
    if world > 1 and not args.no_batch:
        # Every rank takes part (collectives); the batch is split across ranks.
        out["batch"] = batch_metric_sharded(args.precision, rank, world)
    if world == 1 and rank == 0 and not args.no_cpu_baseline:
        try:
            out["cpu_baseline"] = cpu_baseline(n, ops)
        except Exception as e:
            out["cpu_baseline"] = {"value": None, "unit": "GB/s", "kind": "reference",
                                   "sample": f"failed: {e}"}
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out))


def timed_sweeps(n, ops, dtype, steps, warmup, mats=None):
    """Runs the circuit `steps` times after `warmup` untimed runs on a fresh
    state (every gate as a dense matrix, as the benchmark submits them);
    returns (state, ms per step, sweeps per step, ms per sweep launch)."""
    import torch

    from snuqs_b200 import capi, circuits

    mats = mats or [circuits.op_matrix(op, capi.gate_matrix) for op in ops]
    stream = torch.cuda.current_stream().cuda_stream
    st = capi.State(n, dtype, stream=stream)

    def step():
        st.init_basis(0)
        for op, m in zip(ops, mats):
            st.apply_matrix(m, op[1])
        st.flush()

    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    st.sweep_timing()
    st.set_option(capi.SQ_OPT_TIMING, 1)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    for _ in range(steps):
        step()
    ev1.record()
    torch.cuda.synchronize()
    st.set_option(capi.SQ_OPT_TIMING, 0)
    sweep_ms, sweeps = st.sweep_timing()
    return st, ev0.elapsed_time(ev1) / steps, sweeps / steps, sweep_ms / max(1, sweeps)


def sweep_line(name, n, ops, dtype, steps, warmup, note=""):
    from snuqs_b200 import capi

    amp = 16 if dtype == capi.SQ_C128 else 8
    st, ms, sweeps, per = timed_sweeps(n, ops, dtype, steps, warmup)
    peak, _ = measured_peak()
    alg = 2 * amp * (1 << n)
    line = {"workload": name, "qubits": n, "gates": len(ops),
            "precision": "complex128" if dtype == capi.SQ_C128 else "complex64",
            "ms_per_step": round(ms, 3), "fused_sweeps_per_step": sweeps,
            "gates_per_sweep": round(len(ops) / max(1e-9, sweeps), 2),
            "effective_gate_sweep_GBps": round(len(ops) * alg / (ms * 1e-3) / 1e9, 1),
            "per_launch_ms": round(per, 4),
            "roofline_frac": round(alg / (per * 1e-3) / 1e9 / peak, 4) if per > 0 else None,
            "steps": steps, "warmup": warmup}
    if note:
        line["note"] = note
    return st, line


def complex64_metric(st128, n, ops, mats, args):
    """The benchmark circuit on a complex64 state: its time, and its max-abs
    amplitude error and 1 - fidelity against the complex128 result (the
    complex128 path is checked against the reference at 1e-12 by the
    default-path tests)."""
    from snuqs_b200 import capi

    st, line = sweep_line(f"random_mix_{n}q_complex64_{args.gates}g", n, ops, capi.SQ_C64,
                          steps=max(1, min(args.steps, 5)), warmup=2)
    st128.init_basis(0)  # the complex128 state after exactly one run, as the complex64 one
    for op, m in zip(ops, mats):
        st128.apply_matrix(m, op[1])
    st128.flush()
    mx, fl = st.distance(st128)
    st.close()
    line.update({"max_abs_error_vs_complex128": mx, "one_minus_fidelity_vs_complex128": fl})
    return line


def config_metrics():
    """The workload list's other configurations, each timed on its own:
    GHZ-20, QV-28 (complex128 and complex64, with the complex64 error), the
    400-gate random mix at 32 qubits complex128 and 33 qubits complex64."""
    import torch

    from snuqs_b200 import capi, circuits

    out = {}

    def guard(key, fn):
        try:
            out[key] = fn()
        except Exception as e:  # report, keep the rest
            out[key] = {"note": f"failed: {e}"}
        torch.cuda.synchronize()

    def ghz():
        st, line = sweep_line("ghz_20q_complex128", 20, circuits.ghz(20), capi.SQ_C128, 10, 3,
                              note="16 MiB state: L2-resident, the roofline fraction is not an HBM figure")
        psi = st.to_host()
        line["max_abs_error_vs_known_answer"] = float(max(abs(psi[0] - 2 ** -0.5), abs(psi[-1] - 2 ** -0.5),
                                                          np.abs(psi[1:-1]).max()))
        st.close()
        return line

    def qv():
        ops = circuits.quantum_volume(28, 28, seed=28)
        a, la = sweep_line("quantum_volume_28q_d28_complex128", 28, ops, capi.SQ_C128, 5, 2)
        b, lb = sweep_line("quantum_volume_28q_d28_complex64", 28, ops, capi.SQ_C64, 5, 2)
        mx, fl = b.distance(a)
        lb.update({"max_abs_error_vs_complex128": mx, "one_minus_fidelity_vs_complex128": fl})
        a.close()
        b.close()
        return {"complex128": la, "complex64": lb}

    def mix(n, dtype):
        amp = 16 if dtype == capi.SQ_C128 else 8
        free, _ = torch.cuda.mem_get_info()
        if free < 1.1 * (1 << n) * amp:
            return {"note": f"skipped: {free / 2**30:.0f} GiB free"}
        ops = circuits.random_mix(n, 400, seed=SEED)
        st, line = sweep_line(f"random_mix_{n}q_{'complex128' if amp == 16 else 'complex64'}_400g", n,
                              ops, dtype, 3, 1)
        line["norm2_minus_1"] = st.norm2() - 1.0
        st.close()
        return line

    guard("ghz20", ghz)
    guard("qv28", qv)
    guard("mix32_complex128", lambda: mix(32, capi.SQ_C128))
    guard("mix33_complex64", lambda: mix(33, capi.SQ_C64))
    return out


def qaoa_workload(n=26, p=8, seed=SEED):
    """QAOA MaxCut: seeded random 3-regular graph on n vertices, p layers of
    ZZ(gamma_l) on every edge and RotX(beta_l) on every qubit (2p parameters)."""
    from snuqs_b200 import circuits

    edges = circuits.random_regular_graph(n, 3, seed=seed)
    ops = [("Hadamard", (q,), ()) for q in range(n)]
    for l in range(p):
        ops += [("ZZ", (i, j), (0.0,), (l,)) for i, j in edges]
        ops += [("RotX", (q,), (0.0,), (p + l,)) for q in range(n)]
    theta = np.random.default_rng(seed).uniform(0, np.pi, 2 * p)
    return ops, circuits.maxcut_hamiltonian(n, edges), theta


def adjoint_metric(precision: str, shift: bool = True, keep: dict | None = None):
    """Adjoint gradient (one forward + one fused reverse pass) against the
    parameter-shift rule on the same engine, QAOA MaxCut 26 qubits p = 8:
    the full 1040-evaluation shift gradient is computed and compared
    (shift=False: the adjoint gradient alone)."""
    import torch

    from snuqs_b200 import adjoint, capi

    n, p = 26, 8
    dtype = capi.SQ_C128 if precision == "complex128" else capi.SQ_C64
    amp = 16 if dtype == capi.SQ_C128 else 8
    ops, terms, theta = qaoa_workload(n, p)
    ws = adjoint.Workspace(n, dtype)
    for _ in range(2):
        adjoint.adjoint_gradient(ws, ops, theta, terms, 2 * p)
    reps = 5
    torch.cuda.synchronize()
    l0 = ws.psi.launches()
    t0 = time.perf_counter()
    for _ in range(reps):
        e, g = adjoint.adjoint_gradient(ws, ops, theta, terms, 2 * p)
    t_adj = (time.perf_counter() - t0) / reps
    sweeps = (ws.psi.launches() - l0) / reps
    # Device time of the sweeps of one gradient (CUDA events around every
    # forward and reverse sweep launch), then of the forward sweeps alone.
    torch.cuda.synchronize()
    ws.psi.sweep_timing()
    ws.psi.set_option(capi.SQ_OPT_TIMING, 1)
    adjoint.adjoint_gradient(ws, ops, theta, terms, 2 * p)
    grad_sweep_ms, grad_sweeps = ws.psi.sweep_timing()
    adjoint.energy(ws.psi, ops, theta, terms)
    fwd_ms, fwd = ws.psi.sweep_timing()
    ws.psi.set_option(capi.SQ_OPT_TIMING, 0)
    rev = grad_sweeps - fwd
    rev_ms = grad_sweep_ms - fwd_ms
    # Algorithmic HBM bytes: forward sweeps read+write psi; lambda = H psi
    # reads psi and writes lambda (one Pauli flip group for MaxCut); every
    # reverse sweep reads and writes both states.  (launches per gradient also
    # count lambda = H psi and the energy reduction.)
    alg = (2 * fwd + 2 + 4 * rev) * amp * (1 << n)
    peak, peak_kind = measured_peak()
    # The full parameter-shift gradient (2 evaluations per gate occurrence).
    evals = done = adjoint.count_shift_evaluations(ops)
    if shift:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        g_shift = adjoint.parameter_shift_gradient(ws.psi, ops, theta, terms, 2 * p)
        t_shift = time.perf_counter() - t0
        diff = float(np.abs(np.asarray(g) - np.asarray(g_shift)).max())
    ws.close()
    if keep is not None:
        keep["energy"], keep["gradient"] = e, np.array(g, copy=True)
    out = {"workload": f"qaoa_maxcut_{n}q_p{p}_{precision}", "params": 2 * p,
            "gate_occurrences": evals // 2, "energy": e,
            "adjoint_ms": round(t_adj * 1e3, 3), "adjoint_grads_per_s": round(1.0 / t_adj, 3),
            "launches_per_gradient": sweeps, "forward_sweeps": fwd, "reverse_sweeps": rev,
            "forward_sweeps_ms": round(fwd_ms, 3), "reverse_sweeps_ms": round(rev_ms, 3),
            "reverse_sweep_frac": round(4 * amp * (1 << n) * rev / (rev_ms * 1e-3) / 1e9 / peak, 4)
            if rev_ms > 0 else None,
            "forward_sweep_frac": round(2 * amp * (1 << n) * fwd / (fwd_ms * 1e-3) / 1e9 / peak, 4)
            if fwd_ms > 0 else None,
            "roofline": {"bound": "hbm", "achieved": round(alg / t_adj / 1e9, 1), "peak": peak,
                         "unit": "GB/s", "frac": round(alg / t_adj / 1e9 / peak, 4),
                         "algorithmic_bytes": alg, "peak_source": peak_kind,
                         "note": "whole gradient (host wall clock) over its algorithmic bytes"},
           "timing": "host wall clock around synchronous calls; sweep times are CUDA events around "
                     "each sweep launch"}
    if shift:
        out.update({"param_shift_evals_per_grad": evals, "param_shift_evals_done": done,
                    "param_shift_ms": round(t_shift * 1e3, 1),
                    "param_shift_grads_per_s": round(1.0 / t_shift, 4),
                    "speedup_vs_param_shift": round(t_shift / t_adj, 1),
                    "max_abs_adjoint_minus_shift": diff,
                    "tolerance": 1e-10 if dtype == capi.SQ_C128 else 1e-4,
                    "timing": "host wall clock around synchronous calls; the parameter-shift gradient "
                              "is computed in full (every shifted evaluation) and compared with the "
                              "adjoint one; sweep times are CUDA events around each sweep launch"})
    return out


def vqe_batch_circuits(ncirc: int = 4096, seed: int = SEED):
    """The batched-VQE workload: (sizes, circuit_of(i) -> (n, ops, terms))."""
    from snuqs_b200 import circuits

    rng = np.random.default_rng(seed)
    terms = {n: circuits.random_pauli_hamiltonian(n, 64, seed=seed + n) for n in range(8, 21)}
    sizes = [int(x) for x in rng.integers(8, 21, size=ncirc)]
    angles = [rng.uniform(0, 2 * np.pi, 12 * n) for n in sizes]
    return sizes, lambda i: (sizes[i], circuits.vqe_ansatz(sizes[i], angles[i]), terms[sizes[i]])


def batch_complex64_metric(ref_energies, ncirc: int = 4096, seed: int = SEED):
    """The VQE batch of batch_metric (same seed: same circuits and angles) on
    complex64 states: kernel time (default configuration, median of 3) and
    the energies' max-abs error against the complex128 batch."""
    from snuqs_b200 import capi, circuits

    rng = np.random.default_rng(seed)
    b = capi.Batch(capi.SQ_C64)
    hams = {n: b.add_hamiltonian(n, circuits.random_pauli_hamiltonian(n, 64, seed=seed + n))
            for n in range(8, 21)}
    sizes = rng.integers(8, 21, size=ncirc)
    for n in sizes:
        n = int(n)
        b.add_circuit(n, circuits.vqe_ansatz(n, rng.uniform(0, 2 * np.pi, 12 * n)), hams[n])
    b.run()
    ks = []
    for _ in range(3):
        e = b.run()
        ks.append(b.last_timing()[0])
    groups = b.groups()
    b.close()
    err = np.abs(np.asarray(e) - np.asarray(ref_energies))
    return {"workload": f"vqe_batch_{ncirc}x_8to20q_complex64", "kernel_ms": round(float(np.median(ks)), 3),
            "structure_groups": groups[0], "circuits_in_groups": groups[1],
            "max_abs_energy_error_vs_complex128": float(err.max()),
            "max_rel_energy_error_vs_complex128": float((err / np.maximum(1.0, np.abs(ref_energies))).max())}


def batch_metric_sharded(precision: str, rank: int, world: int, ncirc: int = 4096):
    """The batched-VQE energies split across `world` GPUs (one launch each,
    shares balanced by 2^n work), energies gathered to every rank; time = max
    over ranks of one run (strong scaling: the 4096 circuits are fixed)."""
    import torch
    import torch.distributed as dist

    from snuqs_b200 import capi, sharding

    dtype = capi.SQ_C128 if precision == "complex128" else capi.SQ_C64
    sizes, circuit_of = vqe_batch_circuits(ncirc)
    share = sharding.partition(sizes, world)[rank]
    b = capi.Batch(dtype)
    hams = {}
    for i in share:
        n, ops, terms = circuit_of(i)
        if n not in hams:
            hams[n] = b.add_hamiltonian(n, terms)
        b.add_circuit(n, ops, hams[n])
    b.run()  # plan, allocate, capture
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e = b.run()
    t = torch.tensor([time.perf_counter() - t0, b.last_timing()[0] * 1e-3], device="cuda",
                     dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    energies = sharding.gather_results(e, share, len(sizes), rank, world)
    b.close()
    return {"workload": f"vqe_batch_{ncirc}x_8to20q_{precision}", "circuits": ncirc,
            "ranks": world, "scaling": "strong", "run_ms_max_over_ranks": round(t[0].item() * 1e3, 3),
            "kernel_ms_max_over_ranks": round(t[1].item() * 1e3, 3),
            "energies_per_s": round(ncirc / t[0].item(), 1), "energy_checksum": float(np.sum(energies)),
            "timing": "host wall clock of one sq_batch_run per rank (cached plan), max over ranks"}


def qaoa_batch_metric(precision: str, sets: int = 512, n: int = 16, p: int = 8):
    """Adjoint gradients of `sets` QAOA MaxCut parameter sets (n qubits, p
    layers, 2p parameters) in one batched launch, against the same gradients
    one circuit at a time (sq_adjoint_gradient) and the parameter-shift rule,
    on the same GPU."""
    import torch

    from snuqs_b200 import adjoint, capi

    dtype = capi.SQ_C128 if precision == "complex128" else capi.SQ_C64
    ops, terms, _ = qaoa_workload(n, p)
    thetas = np.random.default_rng(SEED + 1).uniform(0, np.pi, (sets, 2 * p))
    b = capi.Batch(dtype)
    hid = b.add_hamiltonian(n, terms)
    for th in thetas:
        b.add_circuit(n, adjoint.bind(ops, th), hid)
    # The gradient kernel also comes with smaller tiles (SQ_BOPT_TILE_BITS 10
    # for complex128, 11 for complex64); those measured slower (128 vs 117 ms
    # and 106 vs 77 ms generic), so only the default is timed here.
    tiles = (11,) if dtype == capi.SQ_C128 else (12,)
    tried = {}
    for tb in tiles:
        b.set_option(capi.SQ_BOPT_TILE_BITS, tb)
        b.run_gradients(2 * p)  # warm-up
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e, g = b.run_gradients(2 * p)
        tried[tb] = (time.perf_counter() - t0, b.last_timing(), e, g)
    best = min(tried, key=lambda k: tried[k][0])
    t_batch, (kernel_ms, ctas), e, g = tried[best]
    b.close()
    # One circuit at a time, on a sample of the parameter sets.
    ws = adjoint.Workspace(n, dtype)
    adjoint.adjoint_gradient(ws, ops, thetas[0], terms, 2 * p)
    sample = 16
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    worst = 0.0
    for k in range(sample):
        _, gk = adjoint.adjoint_gradient(ws, ops, thetas[k], terms, 2 * p)
        worst = max(worst, float(np.abs(gk - g[k]).max()))
    t_single = (time.perf_counter() - t0) / sample
    adjoint.parameter_shift_gradient(ws.psi, ops, thetas[0], terms, 2 * p, max_evals=4)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    _, done = adjoint.parameter_shift_gradient(ws.psi, ops, thetas[0], terms, 2 * p, max_evals=40)
    t_eval = (time.perf_counter() - t0) / done
    evals = adjoint.count_shift_evaluations(ops)
    ws.close()
    return {"workload": f"qaoa_maxcut_{n}q_p{p}_{sets}sets_{precision}", "params": 2 * p,
            "batch_ms": round(t_batch * 1e3, 3), "batch_kernel_ms": round(kernel_ms, 3), "ctas": ctas,
            "tile_bits": best,
            "batch_kernel_ms_by_tile_bits": {str(k): round(v[1][0], 3) for k, v in tried.items()},
            "batch_grads_per_s": round(sets / t_batch, 1),
            "single_adjoint_ms_per_grad": round(t_single * 1e3, 3),
            "single_adjoint_grads_per_s": round(1.0 / t_single, 1),
            "param_shift_grads_per_s": round(1.0 / (t_eval * evals), 3),
            "batch_vs_single_adjoint": round(t_single * sets / t_batch, 1),
            "batch_vs_param_shift": round(t_eval * evals * sets / t_batch, 1),
            "max_abs_diff_vs_single_adjoint": worst,
            "timing": "host wall clock around synchronous calls (batch: planning + upload + one "
                      f"launch); single-circuit adjoint over {sample} sets; parameter shift "
                      f"extrapolated from {done} evaluations"}


def batch_metric(precision: str, ncirc: int = 4096, seed: int = SEED, keep: dict | None = None,
                 tune: bool = True):
    """Batched VQE energies: ncirc hardware-efficient ansatz circuits with
    qubit counts uniform in 8..20 (6 layers of RY, RZ on every qubit and a CX
    ladder, angles uniform in [0, 2pi)), one 64-term random Pauli-sum
    Hamiltonian per qubit count, one energy per circuit, one launch.  Five
    circuits of every qubit count (65) are checked against the oracle."""
    import oracle
    from snuqs_b200 import capi, circuits

    dtype = capi.SQ_C128 if precision == "complex128" else capi.SQ_C64
    amp = 16 if dtype == capi.SQ_C128 else 8
    rng = np.random.default_rng(seed)
    b = capi.Batch(dtype)
    terms = {n: circuits.random_pauli_hamiltonian(n, 64, seed=seed + n) for n in range(8, 21)}
    hams = {n: b.add_hamiltonian(n, terms[n]) for n in range(8, 21)}
    sizes = rng.integers(8, 21, size=ncirc)
    t0 = time.perf_counter()
    circ_ops = []
    for n in sizes:
        n = int(n)
        ops = circuits.vqe_ansatz(n, rng.uniform(0, 2 * np.pi, 12 * n))
        circ_ops.append(ops)
        b.add_circuit(n, ops, hams[n])
    t_add = time.perf_counter() - t0
    t0 = time.perf_counter()
    b.run()  # plans, compiles the structure groups' kernels, allocates, captures the graph
    t_first = time.perf_counter() - t0
    reps = 3

    def kernel_ms():
        ks = []
        for _ in range(reps):
            e = b.run()
            ks.append(b.last_timing()[0])
        return float(np.median(ks)), e

    k_default, energies = kernel_ms()
    cfg = {"tile_bits": 0, "low_bits": 0, "max_ops": 0, "ctas_per_sm": 0}
    t_tune = 0.0
    k_tuned = k_default
    if tune:
        t0 = time.perf_counter()
        cfg = b.autotune(reps=1)
        t_tune = time.perf_counter() - t0
        k_tuned, energies = kernel_ms()
    if keep is not None:
        keep["energies"] = np.array(energies, copy=True)
    ctas = b.last_timing()[1]
    streamed, sweeps, alg = b.stats()
    groups, grouped = b.groups()
    # Oracle check: the first five circuits of every qubit count.
    picked = []
    for n in range(8, 21):
        picked += [i for i in range(ncirc) if int(sizes[i]) == n][:5 if tune else 0]
    worst = 0.0
    for i in picked:
        n = int(sizes[i])
        psi = oracle.run_ops(circ_ops[i], n, use_ref=True)
        want = oracle.expectation_indexed(psi, n, terms[n])
        worst = max(worst, abs(float(energies[i]) - want) / max(1.0, abs(want)))
    # A VQE iteration: new angles for every circuit, then one run (planning,
    # upload and the graph launch are all inside the timed call).
    t_run = 0.0
    for _ in range(reps):
        for cid, n in enumerate(sizes):
            b.set_angles(cid, rng.uniform(0, 2 * np.pi, 12 * int(n)))
        t0 = time.perf_counter()
        b.run()
        t_run += time.perf_counter() - t0
    t_run /= reps
    b.close()
    peak, peak_kind = measured_peak()
    amps = int(sum(1 << int(n) for n in sizes))
    return {"workload": f"vqe_batch_{ncirc}x_8to20q_{precision}", "circuits": ncirc,
            "total_amplitudes": amps, "kernel_ms": round(k_tuned, 3),
            "kernel_ms_default_config": round(k_default, 3),
            "autotuned": {k: cfg[k] for k in ("tile_bits", "low_bits", "max_ops", "ctas_per_sm")},
            "autotune_s": round(t_tune, 2),
            "run_ms": round(t_run * 1e3, 3),
            "energies_per_s": round(ncirc / t_run, 1),
            "energies_per_s_kernel": round(ncirc / (k_tuned * 1e-3), 1),
            "ctas": ctas, "add_circuits_s": round(t_add, 3),
            "structure_groups": groups, "circuits_in_groups": grouped,
            "first_run_s": round(t_first, 2),
            "streamed_circuits": streamed, "streamed_sweeps": sweeps,
            "roofline": {"bound": "hbm", "achieved": round(alg / (k_tuned * 1e-3) / 1e9, 1),
                         "peak": peak, "unit": "GB/s",
                         "frac": round(alg / (k_tuned * 1e-3) / 1e9 / peak, 4),
                         "algorithmic_bytes": alg, "peak_source": peak_kind,
                         "note": "streamed circuits' sweeps (read + write) and one energy read each, "
                                 "over the batch's kernel time (circuits held in shared memory move "
                                 "no HBM bytes)"},
            "oracle_checked_circuits": len(picked),
            "max_rel_error_vs_oracle": worst,
            "tolerance": 1e-10 if dtype == capi.SQ_C128 else 1e-4,
            "timing": "run_ms = host wall clock of sq_batch_run after new angles for every "
                      "circuit (planning + upload + one graph launch); kernel_ms = CUDA events "
                      "around the batch's kernels (median of 3)"}


def e2e(n, ops, args, amp, shots: int = 1_000_000, precision: str | None = None):
    """Same metric through the reference-facing `_C` drop-in, as a shot-based
    Braket task drives it (simulation.py: initialize_basis_z, one
    functionals.apply per gate, then retrieve_samples): each step applies the
    circuit and returns `shots` measurement samples -- the step's uniforms go
    to the device, only the shot indices come back (functionals.sample).
    Every step is timed, K steps as the device-timed line.  The same with the
    StateVector result (the whole state copied to a pinned host buffer) is
    reported beside it."""
    import torch

    from snuqs_b200 import _C

    G = _C.operation.gate_operations
    prec = precision or args.precision
    try:
        sv = _C.result_types.StateVector(_C.DeviceType.CUDA, n, prec)
    except Exception as e:
        return {"value": None, "unit": "GB/s", "note": f"e2e skipped: {e}"}
    gops = [G.Unitary(list(op[1]), op[3]) if op[0] == "Unitary" else
            getattr(G, op[0])(list(op[1]), *op[2]) for op in ops]
    h2d = sum(16 * (1 << (2 * len(g.targets))) for g in gops)
    steps = args.steps
    rng = np.random.default_rng(SEED + 7)
    uniforms = [rng.random(shots) for _ in range(steps + 1)]

    def one(u):
        _C.functionals.initialize_basis_z(sv)
        for g in gops:
            _C.functionals.apply(sv, g, n, g.targets)
        return _C.functionals.sample(sv, u)

    one(uniforms[-1])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for s in range(steps):
        samples = one(uniforms[s])
    t = (time.perf_counter() - t0) / steps
    out = {"value": round(args.gates * 2 * amp * (1 << n) / t / 1e9, 2), "unit": "GB/s",
           "h2d_bytes_per_step": h2d + shots * 8, "d2h_bytes_per_step": shots * 8,
           "ms_per_step": round(t * 1e3, 2), "steps": steps, "precision": prec, "shots": shots,
           "samples_checksum": int(np.sum(samples.astype(np.uint64) % np.uint64(1 << 20))),
           "path": "_C.functionals.apply per gate + functionals.sample (shot indices to the host)",
           "timing": "host wall clock around synchronous steps"}
    # The StateVector result: the whole state to pinned host memory per step.
    try:
        host = _C.result_types.StateVector(n, True, prec)
        sv_steps = max(1, min(steps, 3))

        def one_sv():
            _C.functionals.initialize_basis_z(sv)
            for g in gops:
                _C.functionals.apply(sv, g, n, g.targets)
            host.copy(sv)
            return np.array(host, copy=False)[0]

        one_sv()
        t0 = time.perf_counter()
        for _ in range(sv_steps):
            one_sv()
        tsv = (time.perf_counter() - t0) / sv_steps
        out["state_vector_result"] = {
            "value": round(args.gates * 2 * amp * (1 << n) / tsv / 1e9, 2), "unit": "GB/s",
            "ms_per_step": round(tsv * 1e3, 2), "steps": sv_steps, "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": (1 << n) * amp,
            "path": "_C.functionals.apply per gate + StateVector.copy to pinned host"}
        del host
    except Exception as e:  # pinned allocation can fail on small hosts
        out["state_vector_result"] = {"note": f"skipped: {e}"}
    del sv
    return out


def cpu_baseline(n, ops):
    """The reference CPU path on a bounded, representative sample of the
    same workload: every 10th gate of the circuit in the reference's
    pseudo-sort order (40 of the 400 gates, the mix's 1-, 2- and 3-qubit
    gates in their proportions), one cpu::applyGate each."""
    import oracle

    if not host_ram_ok(n):
        return {"value": None, "unit": "GB/s", "kind": "reference",
                "sample": f"skipped: host RAM below 2.5x the {n}-qubit state"}
    order = pseudo_sorted(ops)
    sample = order[::10]
    psi = np.zeros(1 << n, dtype=np.complex128)
    oracle.ref_initialize_basis_z(psi, n)
    ref_apply(psi, n, sample[0])  # first touch of the state's pages
    t0 = time.perf_counter()
    for op in sample:
        ref_apply(psi, n, op)
    secs = time.perf_counter() - t0
    threads = oracle.ref().ref_max_threads()
    return {"value": round(len(sample) * 2 * AMP_BYTES * (1 << n) / secs / 1e9, 3), "unit": "GB/s",
            "cores": threads, "kind": "reference",
            "sample": f"{len(sample)} of the {len(ops)} gates of the same {n}-qubit circuit (every "
                      f"10th in the reference's pseudo-sort order), {secs:.1f} s, OMP threads {threads}"}


if __name__ == "__main__":
    main()
