"""Batched adjoint gradients (sq_batch_run_gradients): the energies and the
gradients of many parametrised circuits of uneven sizes, computed in one
persistent launch, against the single-circuit adjoint gradient
(sq_adjoint_gradient, itself checked against finite differences and the
parameter-shift rule).  complex128: 1e-10; complex64 against the complex128
reference: 1e-4."""
import numpy as np
import pytest

from snuqs_b200 import adjoint, capi, circuits
from tests.test_adjoint_cpu import random_param_circuit

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _gpu(cuda_required):
    yield


def qaoa(n, p, seed):
    edges = circuits.random_regular_graph(n, 3, seed=seed)
    ops = [("Hadamard", (q,), ()) for q in range(n)]
    for l in range(p):
        ops += [("ZZ", (i, j), (0.0,), (l,)) for i, j in edges]
        ops += [("RotX", (q,), (0.0,), (p + l,)) for q in range(n)]
    return ops, circuits.maxcut_hamiltonian(n, edges), 2 * p


def cases(seed):
    rng = np.random.default_rng(seed)
    out = []
    specs = [("qaoa", 6), ("random", 5), ("qaoa", 8), ("random", 9), ("qaoa", 12),
             ("random", 13), ("qaoa", 14), ("qaoa", 16), ("random", 7)]
    for i, (kind, n) in enumerate(specs):
        if kind == "qaoa":
            ops, terms, npar = qaoa(n, 3, seed=i)
        else:
            npar = 6
            ops = random_param_circuit(n, 40, npar, seed + i)
            terms = circuits.random_pauli_hamiltonian(n, 12, seed=seed + i)
        theta = rng.uniform(-3, 3, npar)
        out.append((n, ops, theta, terms, npar))
    return out


def reference(n, ops, theta, terms, npar):
    ws = adjoint.Workspace(n, capi.SQ_C128)
    e, g = adjoint.adjoint_gradient(ws, ops, theta, terms, npar)
    ws.close()
    return e, g


def run_batch(dtype, cs, n_params):
    b = capi.Batch(dtype)
    ids = []
    for n, ops, theta, terms, _ in cs:
        ids.append(b.add_circuit(n, adjoint.bind(ops, theta), b.add_hamiltonian(n, terms)))
    e, g = b.run_gradients(n_params)
    return b, ids, e, g


@pytest.mark.parametrize("dtype,tol", [(capi.SQ_C128, 1e-10), (capi.SQ_C64, 1e-4)])
def test_batch_gradients_match_single_circuit_adjoint(dtype, tol):
    cs = cases(3)
    n_params = max(c[4] for c in cs)
    b, ids, e, g = run_batch(dtype, cs, n_params)
    for cid, (n, ops, theta, terms, npar) in zip(ids, cs):
        e_ref, g_ref = reference(n, ops, theta, terms, npar)
        assert abs(e[cid] - e_ref) <= tol * max(1.0, abs(e_ref)), (n, e[cid], e_ref)
        assert np.abs(g[cid, :npar] - g_ref).max() <= tol * max(1.0, np.abs(g_ref).max()), n
        assert np.all(g[cid, npar:] == 0.0)
    b.close()


def test_batch_gradient_energies_match_batch_run():
    cs = cases(7)
    n_params = max(c[4] for c in cs)
    b, ids, e, _ = run_batch(capi.SQ_C128, cs, n_params)
    e2 = b.run()
    assert np.abs(e - e2).max() <= 1e-11
    # A second gradient run reuses the buffers and gives the same numbers.
    e3, _ = b.run_gradients(n_params)
    assert np.abs(e - e3).max() <= 1e-12
    b.close()


def test_batch_gradient_parameter_index_checked():
    n = 6
    ops, terms, npar = qaoa(n, 2, seed=1)
    b = capi.Batch(capi.SQ_C128)
    b.add_circuit(n, adjoint.bind(ops, np.ones(npar)), b.add_hamiltonian(n, terms))
    with pytest.raises(capi.SqError, match="n_params"):
        b.run_gradients(npar - 1)
    b.close()


@pytest.mark.parametrize("dtype,tiles,tol", [(capi.SQ_C128, (10, 11), 1e-10), (capi.SQ_C64, (11, 12), 1e-4)])
def test_batch_gradient_tile_sizes_agree(dtype, tiles, tol):
    cs = cases(11)
    n_params = max(c[4] for c in cs)
    b = capi.Batch(dtype)
    for n, ops, theta, terms, _ in cs:
        b.add_circuit(n, adjoint.bind(ops, theta), b.add_hamiltonian(n, terms))
    res = []
    for tb in tiles:
        b.set_option(capi.SQ_BOPT_TILE_BITS, tb)
        res.append(b.run_gradients(n_params))
    assert np.abs(res[0][0] - res[1][0]).max() <= tol
    assert np.abs(res[0][1] - res[1][1]).max() <= tol * max(1.0, np.abs(res[0][1]).max())
    b.close()


@pytest.mark.parametrize("dtype,n,tol", [(capi.SQ_C128, 14, 1e-10), (capi.SQ_C64, 14, 1e-4)])
def test_uniform_batch_jit_kernel_matches_generic(dtype, n, tol, monkeypatch):
    """Many parameter sets of one circuit (every plan has one structure): the
    JIT-specialised batched-gradient kernel against the generic one."""
    ops, terms, npar = qaoa(n, 2, seed=4)
    thetas = np.random.default_rng(9).uniform(-3, 3, (24, npar))
    res = {}
    for jit in ("1", "0"):
        monkeypatch.setenv("SQ_JIT", jit)
        b = capi.Batch(dtype)
        hid = b.add_hamiltonian(n, terms)
        for th in thetas:
            b.add_circuit(n, adjoint.bind(ops, th), hid)
        before = capi.jit_info()[1]
        res[jit] = b.run_gradients(npar)
        if jit == "1":
            assert capi.jit_info()[1] > before, "the JIT batched-gradient kernel did not run"
        b.close()
    assert np.abs(res["1"][0] - res["0"][0]).max() <= tol
    assert np.abs(res["1"][1] - res["0"][1]).max() <= tol * max(1.0, np.abs(res["0"][1]).max())
    e_ref, g_ref = reference(n, ops, thetas[5], terms, npar)
    assert abs(res["1"][0][5] - e_ref) <= tol * max(1.0, abs(e_ref))
