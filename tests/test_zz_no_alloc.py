"""sq_expect_pauli_noalloc: the Pauli expectation for callers that cannot
allocate device memory (graph capture, pool-owned devices, raw state
pointers).  It must give the same value as sq_expect_pauli, call after call,
although both calls share the library's one fixed scratch array.

This file is collected last on purpose, and passes alone or after the rest."""
import ctypes

import numpy as np
import pytest

from snuqs_b200 import capi, circuits

pytestmark = pytest.mark.gpu


def _noalloc(state_ptr, n, dtype, terms, out):
    flat = "".join(p for _, p in terms).encode()
    w = np.ascontiguousarray([x for x, _ in terms], dtype=np.float64)
    capi.check(capi.lib().sq_expect_pauli_noalloc(
        ctypes.c_void_p(state_ptr), n, dtype, flat, w.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
        len(terms), ctypes.c_void_p(out.data_ptr()), None))


@pytest.mark.parametrize("dtype,tol", [(capi.SQ_C128, 1e-12), (capi.SQ_C64, 1e-5)])
def test_noalloc_matches_allocating_entry_point(cuda_required, dtype, tol):
    import torch

    n = 16
    st = capi.State(n, dtype)
    st.init_basis(0)
    st.apply_ops(circuits.random_mix(n, 200, seed=5))
    st.flush()
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    # Two calls in a row, each against the existing entry point; the second
    # uses a different Hamiltonian so stale scratch contents would show.
    for seed, nterms in [(1, 64), (2, 9)]:
        terms = circuits.random_pauli_hamiltonian(n, nterms, seed=seed)
        want = st.expectation(terms)
        _noalloc(st.data_ptr(), n, dtype, terms, out)
        torch.cuda.synchronize()
        got = float(out.item())
        assert abs(got - want) <= tol * max(1.0, abs(want)), (seed, got, want)
    st.close()


def test_noalloc_rejects_oversized_requests(cuda_required):
    import torch

    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    st = capi.State(4)
    st.init_basis(0)
    terms = [(1.0, "ZZZZ")] * 1025
    with pytest.raises(capi.SqError) as e:
        _noalloc(st.data_ptr(), 4, capi.SQ_C128, terms, out)
    assert e.value.status == capi.SQ_ERR_UNSUPPORTED
    st.close()
