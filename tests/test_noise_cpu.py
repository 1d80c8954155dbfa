"""Kraus channels without a GPU: every channel is trace preserving, the
superoperator reproduces sum K rho K^H, and invalid parameters raise."""
import numpy as np
import pytest

from snuqs_b200 import noise_operations as no

CHANNELS = [no.BitFlip([0], 0.1), no.PhaseFlip([0], 0.2), no.PauliChannel([0], 0.1, 0.2, 0.3),
            no.Depolarizing([0], 0.4), no.TwoQubitDepolarizing([0, 1], 0.5),
            no.TwoQubitDephasing([1, 0], 0.3), no.TwoQubitPauliChannel([0, 1], {"XI": 0.1, "YZ": 0.2}),
            no.AmplitudeDamping([0], 0.6), no.GeneralizedAmplitudeDamping([0], 0.3, 0.7),
            no.PhaseDamping([0], 0.45)]


@pytest.mark.parametrize("ch", CHANNELS, ids=lambda c: type(c).__name__)
def test_trace_preserving_and_superoperator(ch):
    ks = ch.matrices
    d = ks[0].shape[0]
    assert np.allclose(sum(k.conj().T @ k for k in ks), np.eye(d), atol=1e-14)
    rng = np.random.default_rng(0)
    a = rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d))
    rho = a @ a.conj().T
    rho /= np.trace(rho)
    want = sum(k @ rho @ k.conj().T for k in ks)
    got = (ch.superoperator() @ rho.reshape(-1)).reshape(d, d)
    assert np.allclose(got, want, atol=1e-14)


def test_invalid_channels_raise():
    with pytest.raises(ValueError):
        no.BitFlip([0], 1.5)
    with pytest.raises(ValueError):
        no.PauliChannel([0], 0.5, 0.4, 0.3)
    with pytest.raises(ValueError):
        no.TwoQubitDepolarizing([0, 0], 0.1)
    with pytest.raises(ValueError):
        no.Kraus([0], [np.eye(2), np.eye(2)])
    with pytest.raises(ValueError):
        no.TwoQubitPauliChannel([0, 1], {"II": 0.1})
