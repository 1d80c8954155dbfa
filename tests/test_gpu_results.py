"""Result kernels on the GPU against the oracle, through the C ABI: device
measurement sampling (bit-identical shot indices for fixed uniforms),
amplitude lookup, marginal probabilities, Pauli-sum variance, and the
out-of-memory path of state creation."""
import numpy as np
import pytest

import oracle
from snuqs_b200 import capi, circuits

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _gpu(cuda_required):
    yield


def _state(n, ops, dtype=capi.SQ_C128):
    st = capi.State(n, dtype)
    st.init_basis(0)
    st.apply_ops(ops)
    st.flush()
    return st


@pytest.mark.parametrize("n", [3, 12, 13, 18, 21])
@pytest.mark.parametrize("dtype", [capi.SQ_C128, capi.SQ_C64])
def test_sampling_is_the_oracle_inverse_cdf(n, dtype):
    ops = circuits.random_all_gates(n, 80, seed=300 + n)
    st = _state(n, ops, dtype)
    psi = st.to_host()
    rng = np.random.default_rng(n)
    u = rng.random(50000)
    u[:4] = [0.0, 0.5, np.nextafter(1.0, 0.0), 1e-300]
    got = st.sample(u)
    want = oracle.sample_inverse_cdf(psi, u)
    assert np.array_equal(got, want)
    # Two calls in a row reuse the state's scratch.
    assert np.array_equal(st.sample(u[::-1]), want[::-1])
    st.close()


def test_sampling_known_answers():
    n = 16
    st = _state(n, circuits.ghz(n))
    idx = st.sample(np.random.default_rng(1).random(10000))
    assert set(np.unique(idx).tolist()) == {0, (1 << n) - 1}
    assert abs(np.mean(idx == 0) - 0.5) < 0.03
    st.init_basis(12345)
    assert np.all(st.sample(np.linspace(0, 0.999, 777)) == 12345)
    st.close()


def test_sampling_30_qubits_one_million_shots():
    """The headline state size: 10^6 shots of a 30-qubit complex128 state,
    checked against the oracle walk on a sample of the shots."""
    import torch

    free, _ = torch.cuda.mem_get_info()
    if free < 20 * (1 << 30):
        pytest.skip("needs 20 GiB free device memory")
    n = 30
    ops = [("Hadamard", (q,), ()) for q in range(n)] + circuits.random_mix(n, 40, seed=9)
    st = _state(n, ops)
    u = np.random.default_rng(2).random(1_000_000)
    got = st.sample(u)
    assert got.max() < (1 << n)
    psi = st.to_host()
    sel = np.arange(0, u.size, 997)
    assert np.array_equal(got[sel], oracle.sample_inverse_cdf(psi, u[sel]))
    st.close()


@pytest.mark.parametrize("dtype", [capi.SQ_C128, capi.SQ_C64])
def test_amplitudes_and_marginals(dtype):
    n = 14
    st = _state(n, circuits.random_all_gates(n, 200, seed=3), dtype)
    psi = st.to_host()
    rng = np.random.default_rng(5)
    idx = rng.integers(0, 1 << n, size=500)
    amp = st.amplitudes(idx)
    assert np.array_equal(amp, psi[idx].astype(np.complex128))
    for qs in ([0], [n - 1], [3, 1], [0, 5, 9, 13], list(range(n)), [7, 2, 11, 4, 0, 12]):
        want = oracle.marginal_probabilities(psi, n, qs)
        tol = 1e-12 if dtype == capi.SQ_C128 else 1e-6
        assert np.abs(st.marginal_probabilities(qs) - want).max() <= tol, qs
    with pytest.raises(capi.SqError) as e:
        st.amplitudes([1 << n])
    assert e.value.status == capi.SQ_ERR_INVALID
    with pytest.raises(capi.SqError):
        st.marginal_probabilities([2, 2])
    st.close()


@pytest.mark.parametrize("dtype,tol", [(capi.SQ_C128, 1e-12), (capi.SQ_C64, 1e-5)])
def test_variance(dtype, tol):
    for n in (6, 15):
        ops = circuits.random_all_gates(n, 150, seed=n)
        ref = oracle.run_ops(ops, n)
        st = _state(n, ops, dtype)
        for terms in (circuits.random_pauli_hamiltonian(n, 12, seed=n),
                      [(1.0, "Z" * n)], [(2.5, "X" + "Y" * (n - 1))],
                      [(0.7, "Z" + "I" * (n - 1)), (-0.3, "I" * (n - 1) + "Z"), (0.2, "X" * n)]):
            want = oracle.variance(ref, n, terms)
            got = st.variance(terms)
            assert abs(got - want) <= tol * max(1.0, abs(want)), (n, terms[:2], got, want)
        st.close()


def test_state_larger_than_the_device_is_oom_and_engine_stays_usable():
    with pytest.raises(capi.SqError) as e:
        capi.State(36)  # 1 TiB of complex128
    assert e.value.status == capi.SQ_ERR_OOM
    n = 10
    ops = circuits.random_all_gates(n, 50, seed=1)
    st = _state(n, ops)
    assert np.abs(st.to_host() - oracle.run_ops(ops, n)).max() <= 1e-12
    st.close()


def test_state_distance_reports_complex64_error():
    n = 16
    ops = circuits.random_mix(n, 300, seed=16)
    a = _state(n, ops, capi.SQ_C128)
    b = _state(n, ops, capi.SQ_C64)
    pa, pb = a.to_host(), b.to_host().astype(np.complex128)
    mx, fl = b.distance(a)
    assert abs(mx - np.abs(pa - pb).max()) <= 1e-12
    want_fl = 1 - abs(np.vdot(pb, pa)) ** 2 / (np.vdot(pa, pa).real * np.vdot(pb, pb).real)
    assert abs(fl - want_fl) <= 1e-12
    assert mx <= 1e-5 and fl <= 1e-9
    assert a.distance(a) == (0.0, pytest.approx(0.0, abs=1e-15))
    a.close()
    b.close()


def test_host_sampling_through_the_pybind_layer():
    """_C.functionals.sample (sq_sample_host): host uniforms in, shot indices
    out, the same indices as the oracle's walk."""
    from snuqs_b200 import _C

    n = 15
    ops = circuits.random_all_gates(n, 120, seed=15)
    G = _C.operation.gate_operations
    sv = _C.result_types.StateVector(_C.DeviceType.CUDA, n)
    _C.functionals.initialize_basis_z(sv)
    for op in ops:
        g = getattr(G, op[0])(list(op[1]), *op[2])
        _C.functionals.apply(sv, g, n, list(op[1]))
    u = np.random.default_rng(3).random(30000)
    got = _C.functionals.sample(sv, u)
    want = oracle.sample_inverse_cdf(oracle.run_ops(ops, n), u)
    assert got.dtype == np.uint64 and np.array_equal(got, want)
