"""C ABI checks that need no GPU: the library loads, exports every entry
point include/snuqs_b200.h declares, builds the reference's gate matrices,
and reports errors as status codes instead of exiting."""
import os
import re

import numpy as np
import pytest

import oracle
from snuqs_b200 import capi
from tests.conftest import ROOT


def declared_functions():
    src = open(os.path.join(ROOT, "include", "snuqs_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(sq_[a-z0-9_]+)\s*\(", src)))


def test_header_declarations_are_bound_and_exported():
    names = declared_functions()
    assert len(names) >= 40
    lib = capi.lib()
    for n in names:
        assert hasattr(lib, n), n
        assert n in capi.SIGNATURES, n


def test_version():
    assert b"sm_100a" in capi.lib().sq_version()


@pytest.mark.parametrize("name", capi.GATE_NAMES)
def test_gate_matrices_match_reference(name):
    na = oracle.gate_num_angles(name)
    for a in [(0.3, 1.1, -2.0), (np.pi, np.pi / 2, 0.0)]:
        got = capi.gate_matrix(name, a[:na])
        want = oracle.gate_matrix(name, a[:na])
        if name in oracle.REFERENCE_GATES:
            assert np.array_equal(got, oracle.ref_gate_matrix(name, a[:na])), name
        assert np.allclose(got, want, atol=1e-15), name
        d = got.shape[0]
        assert np.allclose(got @ got.conj().T, np.eye(d), atol=1e-14), name


def test_bad_gate_is_an_error_not_an_exit():
    with pytest.raises(capi.SqError) as e:
        capi.gate_matrix("RotX", ())  # missing angle
    assert e.value.status == capi.SQ_ERR_INVALID


def test_no_gpu_state_create_fails_cleanly():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(capi.SqError) as e:
        capi.State(4)
    assert e.value.status in (capi.SQ_ERR_CUDA, capi.SQ_ERR_OOM)


PARAM_GATES = ["PhaseShift", "CPhaseShift", "CPhaseShift00", "CPhaseShift01", "CPhaseShift10",
               "RotX", "RotY", "RotZ", "PSwap", "XY", "XX", "YY", "ZZ", "U", "GPhase", "PRx"]


@pytest.mark.parametrize("name", PARAM_GATES)
def test_gate_derivatives_match_finite_differences(name):
    rng = np.random.default_rng(11)
    na = oracle.gate_num_angles(name)
    for _ in range(3):
        a = rng.uniform(-3, 3, size=na)
        for p in range(na):
            d = capi.gate_matrix_derivative(name, a, p)
            h = 1e-5
            ap, am = a.copy(), a.copy()
            ap[p] += h
            am[p] -= h
            fd = (capi.gate_matrix(name, ap) - capi.gate_matrix(name, am)) / (2 * h)
            assert np.abs(d - fd).max() < 1e-9, (name, p)


def test_derivative_of_fixed_gate_is_an_error():
    with pytest.raises(capi.SqError):
        capi.gate_matrix_derivative("CX", (), 0)
