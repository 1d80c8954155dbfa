"""sq_expect_pauli_noalloc: the Pauli expectation for callers that cannot
allocate device memory -- code recording a CUDA graph (an allocation would
break the capture), applications whose memory pool owns the whole device, and
callers that hold only a raw device pointer to a state.  It must give the same
value as sq_expect_pauli and as the oracle, call after call, although every
call shares the library's one fixed scratch array.

This file is collected last on purpose, and passes alone or after the rest."""
import ctypes

import numpy as np
import pytest

import oracle
from snuqs_b200 import capi, circuits

pytestmark = pytest.mark.gpu


def _noalloc(state_ptr, n, dtype, terms, out, stream=None):
    flat = "".join(p for _, p in terms).encode()
    w = np.ascontiguousarray([x for x, _ in terms], dtype=np.float64)
    capi.check(capi.lib().sq_expect_pauli_noalloc(
        ctypes.c_void_p(state_ptr), n, dtype, flat, w.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
        len(terms), ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream) if stream else None))


@pytest.mark.parametrize("dtype,tol", [(capi.SQ_C128, 1e-12), (capi.SQ_C64, 1e-5)])
def test_noalloc_matches_allocating_entry_point(cuda_required, dtype, tol):
    import torch

    n = 16
    ops = circuits.random_mix(n, 200, seed=5)
    ref = oracle.run_ops(ops, n)
    st = capi.State(n, dtype)
    st.init_basis(0)
    st.apply_ops(ops)
    st.flush()
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    # Two calls in a row, each against the existing entry point and the
    # oracle; the second uses a different Hamiltonian so stale scratch
    # contents would show.
    for seed, nterms in [(1, 64), (2, 9)]:
        terms = circuits.random_pauli_hamiltonian(n, nterms, seed=seed)
        want = st.expectation(terms)
        exact = oracle.expectation(ref, n, terms)
        _noalloc(st.data_ptr(), n, dtype, terms, out)
        torch.cuda.synchronize()
        got = float(out.item())
        assert abs(got - want) <= tol * max(1.0, abs(want)), (seed, got, want)
        assert abs(got - exact) <= tol * max(1.0, abs(exact)), (seed, got, exact)
    st.close()


def test_noalloc_inside_a_captured_graph(cuda_required):
    """One eager call sets the device up; then the call is recorded into a
    CUDA graph and replayed on a state held in a plain torch tensor."""
    import torch

    n = 14
    ops = circuits.random_all_gates(n, 120, seed=8)
    ref = oracle.run_ops(ops, n)
    psi = torch.from_numpy(ref.copy()).cuda()
    terms = circuits.random_pauli_hamiltonian(n, 24, seed=3)
    exact = oracle.expectation(ref, n, terms)
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    _noalloc(psi.data_ptr(), n, capi.SQ_C128, terms, out)  # set-up outside the capture
    torch.cuda.synchronize()
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        g.capture_begin()
        _noalloc(psi.data_ptr(), n, capi.SQ_C128, terms, out, stream=s.cuda_stream)
        g.capture_end()
    for _ in range(2):
        out.zero_()
        g.replay()
        torch.cuda.synchronize()
        assert abs(float(out.item()) - exact) <= 1e-12 * max(1.0, abs(exact))


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
    # 257 distinct X masks: one group each, one more than the array allows.
    n = 9
    st = capi.State(n)
    st.init_basis(0)
    masks = [format(m, f"0{n}b") for m in range(257)]
    terms = [(1.0, "".join("X" if c == "1" else "Z" for c in m)) for m in masks]
    with pytest.raises(capi.SqError) as e:
        _noalloc(st.data_ptr(), n, capi.SQ_C128, terms, out)
    assert e.value.status == capi.SQ_ERR_UNSUPPORTED
    # The library stays usable after the rejections.
    _noalloc(st.data_ptr(), n, capi.SQ_C128, terms[:256], out)
    torch.cuda.synchronize()
    assert abs(float(out.item()) - st.expectation(terms[:256])) <= 1e-12
    st.close()
