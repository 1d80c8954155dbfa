"""Parity of the JIT-specialised sweep kernels (SQ_OPT_JIT = 1) against the
oracle and against the generic sweep kernel, through the C ABI.  Tolerances
as in test_gpu_parity: complex128 max-abs <= 1e-12; complex64 max-abs
<= 1e-5 against the complex128 oracle."""
import numpy as np
import pytest

import oracle
from snuqs_b200 import capi, circuits

pytestmark = pytest.mark.gpu
TOL128 = 1e-12
TOL64 = 1e-5


@pytest.fixture(scope="module", autouse=True)
def _gpu(cuda_required):
    import torch

    torch.cuda.init()
    assert capi.jit_info()[0], "NVRTC must be loadable on the GPU box"
    yield


def run(ops, n, dtype=capi.SQ_C128, jit=1, psi0=None, tile_bits=12, low_bits=0):
    st = capi.State(n, dtype)
    st.set_option(capi.SQ_OPT_JIT, jit)
    st.set_option(capi.SQ_OPT_TILE_BITS, tile_bits)
    st.set_option(capi.SQ_OPT_LOW_BITS, low_bits)
    if psi0 is None:
        st.init_basis(0)
    else:
        st.from_host(psi0)
    st.apply_ops(ops)
    out = st.to_host()
    st.close()
    return out


@pytest.mark.parametrize("dtype", [capi.SQ_C128, capi.SQ_C64])
@pytest.mark.parametrize("n", [12, 16])
def test_all_gates_against_oracle(n, dtype):
    ops = circuits.random_all_gates(n, 250, seed=100 + n)
    before = capi.jit_info()[1]
    got = run(ops, n, dtype)
    assert capi.jit_info()[1] > before, "the JIT kernels did not run"
    ref = oracle.run_ops(ops, n)
    tol = TOL128 if dtype == capi.SQ_C128 else TOL64
    assert np.abs(got - ref).max() <= tol


@pytest.mark.parametrize("tile_bits", [7, 10, 12])
def test_tile_sizes_against_oracle(tile_bits):
    n = 14
    ops = circuits.random_mix(n, 200, seed=tile_bits)
    got = run(ops, n, tile_bits=tile_bits)
    assert np.abs(got - oracle.run_ops(ops, n)).max() <= TOL128


def test_quantum_volume_against_oracle():
    n = 12
    ops = circuits.quantum_volume(n, 6, seed=9)
    got = run(ops, n, capi.SQ_C64)
    assert np.abs(got - oracle.run_ops(ops, n)).max() <= TOL64


@pytest.mark.parametrize("dtype", [capi.SQ_C128, capi.SQ_C64])
def test_large_state_matches_generic_kernel(dtype):
    # 24 qubits: controls and diagonal targets outside the tile.
    n = 24
    ops = circuits.random_mix(n, 300, seed=21)
    a = run(ops, n, dtype, jit=1)
    b = run(ops, n, dtype, jit=0)
    tol = 1e-13 if dtype == capi.SQ_C128 else 1e-6
    assert np.abs(a - b).max() <= tol
    a64 = a.astype(np.complex128)
    assert abs(np.vdot(a64, a64).real - 1.0) <= (1e-12 if dtype == capi.SQ_C128 else 1e-4)


def test_cached_kernel_serves_new_angles():
    n = 20
    ops = circuits.random_mix(n, 120, seed=31)
    run(ops, n)
    rng = np.random.default_rng(1)
    ops2 = [(nm, q, tuple(rng.uniform(0.1, 3.0, size=len(a)))) for nm, q, a in ops]
    a = run(ops2, n, jit=1)
    b = run(ops2, n, jit=0)
    assert np.abs(a - b).max() <= 1e-13


@pytest.mark.parametrize("jit", [0, 1])
@pytest.mark.parametrize("low_bits", [2, 3, 4])
def test_low_bits_against_oracle(jit, low_bits):
    n = 16
    ops = circuits.random_all_gates(n, 250, seed=200 + low_bits)
    ref = oracle.run_ops(ops, n)
    got = run(ops, n, capi.SQ_C128, jit=jit, tile_bits=11, low_bits=low_bits)
    assert np.abs(got - ref).max() <= TOL128
    got = run(ops, n, capi.SQ_C64, jit=jit, tile_bits=12, low_bits=low_bits)
    assert np.abs(got - ref).max() <= TOL64


@pytest.mark.parametrize("dtype", [capi.SQ_C128, capi.SQ_C64])
def test_low_bits_large_state_matches_default(dtype):
    n = 24
    ops = circuits.random_mix(n, 300, seed=23)
    a = run(ops, n, dtype, jit=1, low_bits=5)
    b = run(ops, n, dtype, jit=0)
    assert np.abs(a - b).max() <= (1e-13 if dtype == capi.SQ_C128 else 1e-6)


@pytest.mark.parametrize("dtype", [capi.SQ_C128, capi.SQ_C64])
def test_jit_adjoint_matches_generic_adjoint(dtype):
    from snuqs_b200 import adjoint
    from tests.test_adjoint_cpu import random_param_circuit

    edges = circuits.random_regular_graph(20, 3, seed=2)
    qaoa = [("Hadamard", (q,), ()) for q in range(20)]
    for l in range(2):
        qaoa += [("ZZ", (i, j), (0.0,), (l,)) for i, j in edges]
        qaoa += [("RotX", (q,), (0.0,), (2 + l,)) for q in range(20)]
    cases = [(20, qaoa, circuits.maxcut_hamiltonian(20, edges), 4),
             (14, random_param_circuit(14, 40, 6, 5), circuits.random_pauli_hamiltonian(14, 12, seed=5), 6)]
    for n, ops, terms, npar in cases:
        theta = np.random.default_rng(n).uniform(-3, 3, npar)
        res = {}
        for jit in (0, 1):
            ws = adjoint.Workspace(n, dtype)
            ws.psi.set_option(capi.SQ_OPT_JIT, jit)
            before = capi.jit_info()[1]
            res[jit] = adjoint.adjoint_gradient(ws, ops, theta, terms, npar)
            if jit:
                assert capi.jit_info()[1] > before, "the JIT kernels did not run"
            ws.close()
        tol = 1e-10 if dtype == capi.SQ_C128 else 1e-4
        assert abs(res[0][0] - res[1][0]) <= tol
        assert np.abs(res[0][1] - res[1][1]).max() <= tol * max(1.0, np.abs(res[0][1]).max())
