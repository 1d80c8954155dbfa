"""JIT-specialised sweep kernels, without a GPU: the generated CUDA source of
every fused sweep compiles with NVRTC for sm_100a, depends on the circuit's
structure only (angles are kernel parameters, so one compiled kernel serves
every parameter value), and covers every sweep-op kind the planner emits."""
import re

import numpy as np
import pytest

from snuqs_b200 import capi, circuits

pytestmark = pytest.mark.skipif(not capi.jit_info()[0], reason="NVRTC is not available")

OP_ROUTINES = ("op_phase", "op_diag", "op_anti1", "op_swap2", "op_xrot", "op_dense")


def _cases():
    return [
        ("all_gates_14q_c128", 14, circuits.random_all_gates(14, 300, seed=5), capi.SQ_C128),
        ("all_gates_14q_c64", 14, circuits.random_all_gates(14, 300, seed=6), capi.SQ_C64),
        ("random_mix_26q_c128", 26, circuits.random_mix(26, 120, seed=7), capi.SQ_C128),
        ("quantum_volume_12q_c64", 12, circuits.quantum_volume(12, 4, seed=8), capi.SQ_C64),
    ]


@pytest.mark.parametrize("case", _cases(), ids=lambda c: c[0])
def test_generated_sources_compile(case):
    _, n, ops, dtype = case
    srcs = capi.jit_sources(n, ops, dtype)
    assert srcs
    for src in srcs[:12]:
        capi.jit_compile(src)


def test_sources_cover_every_op_kind():
    seen = set()
    for _, n, ops, dtype in _cases():
        for src in capi.jit_sources(n, ops, dtype):
            body = src[src.rindex("sq_jit_sweep"):]
            seen |= {r for r in OP_ROUTINES if r + "<" in body}
            if "gbase & 0x" in body:
                seen.add("global_control")
            if "jb & 0x" in body:
                seen.add("tile_control")
            if "Ph::store(" in body:
                seen.add("direct_store")
            if "Ph::load(" in body or "Ph0::load(" in body:
                seen.add("direct_load")
            if "JitTileMap<" in body:
                seen.add("remapping_store")
            if "Ph::gather_lin(" in body and "jit_sweep_pipe<" in body:
                seen.add("bulk_copy_pipeline")
    # Direct-load sweeps take their tiles through the bulk-copy pipeline by
    # default (SQ_JIT_STAGES=0 brings back the register loads).
    first = "bulk_copy_pipeline" if "bulk_copy_pipeline" in seen else "direct_load"
    assert seen >= set(OP_ROUTINES) | {"global_control", "direct_store", first}, seen


def test_sources_depend_on_structure_not_angles():
    n = 24
    a = circuits.random_mix(n, 150, seed=11)
    rng = np.random.default_rng(3)
    b = [(name, q, tuple(rng.uniform(0.1, 3.0, size=len(ang)))) for name, q, ang in a]
    sa, sb = capi.jit_sources(n, a), capi.jit_sources(n, b)
    assert sa == sb


def test_compile_errors_are_reported():
    with pytest.raises(capi.SqError, match="NVRTC compile failed"):
        capi.jit_compile("extern \"C\" __global__ void sq_jit_sweep() { undefined_name(); }")


def test_kernel_signature():
    src = capi.jit_sources(20, circuits.random_mix(20, 30, seed=2), capi.SQ_C64, limit=1)[0]
    assert re.search(r'extern "C" __global__ void __launch_bounds__\(256, 2\)\s*sq_jit_sweep', src)


SWZ_IMAGES = {  # sweep_kernels.cuh, Swz<Real>::kImage
    capi.SQ_C128: (3, [1, 2, 4, 7, 3, 5, 6, 4, 5, 7, 6, 6]),
    capi.SQ_C64: (4, [1, 2, 4, 8, 14, 11, 7, 13, 10, 15, 6, 10]),
}


def _rank(vectors):
    basis = []
    for v in vectors:
        for b in basis:
            v = min(v, v ^ b)
        if v:
            basis.append(v)
    return len(basis)


@pytest.mark.parametrize("dtype", [capi.SQ_C128, capi.SQ_C64])
def test_lane_placement_is_a_permutation_and_conflict_free(dtype):
    n = 26
    W, img = SWZ_IMAGES[dtype]
    phases = conflict_free = 0
    for src in capi.jit_sources(n, circuits.random_mix(n, 200, seed=13), dtype):
        body = src[src.rindex("sq_jit_sweep"):]
        # Direct-store phases of remapping sweeps place their lanes for a
        # coalesced permuted store (output order), not for the gather.
        permuted = set(re.findall(r"JitPhase<\w+, \d+, TileOut, ([\d, ]+)>", body))
        for mm, args in re.findall(r"JitPhase<\w+, (\d+), Tile, ([\d, ]+)>", body):
            vals = [int(x) for x in args.split(",")]
            m, regs, threads = int(mm), vals[:4], vals[4:]
            assert sorted(regs + threads) == list(range(m))
            if args in permuted:
                continue
            phases += 1
            conflict_free += _rank([img[p] for p in threads[:W]]) == W
    assert phases > 0
    # Every other phase gets independent lane images (direct-load and
    # direct-store phases have ascending lanes from tile position 0, also
    # conflict-free).
    assert conflict_free == phases


def _qaoa(n, p, seed):
    edges = circuits.random_regular_graph(n, 3, seed=seed)
    ops = [("Hadamard", (q,), ()) for q in range(n)]
    for l in range(p):
        ops += [("ZZ", (i, j), (0.3,), (l,)) for i, j in edges]
        ops += [("RotX", (q,), (0.7,), (p + l,)) for q in range(n)]
    return ops


@pytest.mark.parametrize("dtype", [capi.SQ_C128, capi.SQ_C64])
def test_adjoint_sources_compile(dtype):
    from tests.test_adjoint_cpu import random_param_circuit

    cases = [(20, _qaoa(20, 2, seed=1)), (14, random_param_circuit(14, 40, 6, 3))]
    compiled = 0
    for n, ops in cases:
        srcs = capi.jit_sources(n, ops, dtype, adjoint=True)
        assert srcs
        for src in srcs[:6]:
            if src:
                assert "sq_jit_adjoint" in src
                capi.jit_compile(src)
                compiled += 1
    assert compiled > 0


def test_adjoint_inner_products_take_the_pauli_form():
    """Rotation generators (RotX: X, ZZ: Z x Z, RotY: Y) are single Pauli
    strings: their inner products use the four-FMA routines; PhaseShift's
    generator (I - Z)/2 is not and keeps the general routine.  Coefficients of
    the reverse sweeps come from shared memory (no parameter-block reads)."""
    srcs = capi.jit_sources(20, _qaoa(20, 1, seed=2), capi.SQ_C128, adjoint=True)
    body = "".join(s.split("sq_jit_adjoint(")[1] for s in srcs if s)
    assert "inner_dense_pauli<" in body
    # ZZ generators: one at a time, or several from the shared products of a
    # fused diagonal run.
    assert "inner_diag_pauli<" in body or "Pauli-Z inner products from shared products" in body
    assert "Pauli-Z inner products from shared products" in body and "diagonal ops, fused" in body
    assert "inner_dense<" not in body and "inner_diag<" not in body
    assert "ParamCoef<" not in body
    ops = [("Hadamard", (q,), ()) for q in range(20)]
    ops += [("PhaseShift", (q,), (0.2,), (0,)) for q in range(20)]
    ops += [("RotY", (q,), (0.4,), (1,)) for q in range(20)]
    srcs = capi.jit_sources(20, ops, capi.SQ_C128, adjoint=True)
    body = "".join(s.split("sq_jit_adjoint(")[1] for s in srcs if s)
    assert "inner_diag<" in body and "inner_dense_pauli<" in body
    capi.jit_compile(next(s for s in srcs if s))


@pytest.mark.parametrize("dtype,n", [(capi.SQ_C128, 14)])
def test_batch_adjoint_source_compiles(dtype, n):
    from snuqs_b200 import adjoint

    edges = circuits.random_regular_graph(n, 3, seed=3) if n % 2 == 0 else [(i, (i + 1) % n) for i in range(n)]
    ops = [("Hadamard", (q,), ()) for q in range(n)]
    for l in range(2):
        ops += [("ZZ", (i, j), (0.0,), (l,)) for i, j in edges]
        ops += [("RotX", (q,), (0.0,), (2 + l,)) for q in range(n)]
    src = capi.jit_batch_adjoint_source(n, adjoint.bind(ops, [0.3, 0.5, 0.7, 0.9]), dtype)
    assert "sq_jit_batch_adjoint" in src
    capi.jit_compile(src)


@pytest.mark.parametrize("env", ["SQ_JIT_EARLY=1", "SQ_JIT_STAGES=1", "SQ_REMAP=1"])
def test_alternative_tile_loops_compile(env):
    """The early-load and bulk-copy tile loops (off by default) generate
    sources that compile, for both precisions (a subprocess: the switches
    are read once per process)."""
    import os
    import subprocess
    import sys

    code = (
        "import sys; sys.path.insert(0, %r)\n"
        "from snuqs_b200 import capi, circuits\n"
        "for n, dt in ((26, capi.SQ_C128), (24, capi.SQ_C64)):\n"
        "    srcs = capi.jit_sources(n, circuits.random_mix(n, 120, seed=7), dt)\n"
        "    key = %r\n"
        "    assert any(key in s for s in srcs), key\n"
        "    for s in srcs[:3]:\n"
        "        capi.jit_compile(s)\n"
    ) % (os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
         {"SQ_JIT_EARLY": "jit_sweep_early<", "SQ_JIT_STAGES": "jit_sweep_pipe<",
          "SQ_REMAP": "JitTileMap<"}[env.split("=")[0]])
    k, v = env.split("=")
    # Early loads apply to direct-load sweeps; complex64 turns those on with SQ_JIT_DLOAD.
    r = subprocess.run([sys.executable, "-c", code], env={**os.environ, k: v, "SQ_JIT_DLOAD": "1"},
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]


@pytest.mark.parametrize("dtype,n", [(capi.SQ_C128, 16), (capi.SQ_C64, 14)])
def test_multi_state_sources_compile(dtype, n):
    """The multi-state kernels of a batch energy plan (one launch per sweep
    over every state of a structure group) compile; coefficients come from
    the shared-memory copy of each state's block."""
    ops = circuits.vqe_ansatz(n, np.random.default_rng(n).uniform(0, 2 * np.pi, 12 * n))
    srcs = capi.jit_sources(n, ops, dtype, multi=True)
    assert srcs and all("sq_jit_msweep" in s and "MultiParams Q" in s for s in srcs)
    assert not any("ParamCoef<" in s.split("sq_jit_msweep")[1] for s in srcs)
    for s in srcs[:2]:
        capi.jit_compile(s)
    # The first sweep in the form that starts every state from |0...0>.
    z = capi.jit_sources(n, ops, dtype, multi=True, from_zero=True, limit=1)[0]
    assert "zero_state(" in z and "Ph0::load(" not in z.split("sq_jit_msweep")[1]
    capi.jit_compile(z)
