"""Device observables (discoeb_power_amplitudes, discoeb_savgol_log_power, discoeb_power_kaiser,
discoeb_power_multipoles, discoeb_xi_from_power) against the CPU restatement (GPU)."""
import numpy as np
import pytest

from oracle import observables_oracle as OB

pytestmark = pytest.mark.gpu

PARAM = {"A_s": 2.1e-9, "n_s": 0.965, "k_p": 0.05}


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("no CUDA device: the -m gpu tests need a GPU")
    return torch


def _outputs(K=256, seed=2):
    """smooth synthetic output fields: delta_m > 0, theta_m/(aH) < 0"""
    rng = np.random.default_rng(seed)
    k = np.geomspace(1e-4, 2.0, K)
    y = np.zeros((K, 20))
    lk = np.log(k)
    y[:, 4] = 1e3 * (1 + 0.3 * np.sin(3 * lk)) / (1 + (k / 0.02) ** 2) ** 0.8 + rng.uniform(0, 1e-6, K)
    y[:, 5] = -0.5 * y[:, 4] * (1 + 0.1 * np.cos(2 * lk))
    return k, y


def test_gpu_kaiser_and_multipoles_match_oracle(torch_cuda):
    from discoeb_b200.observables import power_Kaiser, power_multipoles
    k, y = _outputs()
    for mu_sampling in (True, False):
        got, mu = power_Kaiser(y=y, kmodes=k, bias=1.6, mu_sampling=mu_sampling, nmu=9, param=PARAM)
        want, mu_ref = OB.power_Kaiser(y, k, 1.6, 9, mu_sampling=mu_sampling, **PARAM)
        np.testing.assert_array_equal(mu, mu_ref)
        np.testing.assert_allclose(got, want, rtol=1e-13)
    got = power_multipoles(y=y, kmodes=k, b=1.6, param=PARAM)
    for g, w in zip(got, OB.power_multipoles(y, k, 1.6, **PARAM)):
        np.testing.assert_allclose(g, w, rtol=1e-12, atol=1e-13 * np.abs(w).max())


def test_gpu_smoothed_power_and_smoothed_kaiser_match_oracle(torch_cuda):
    from discoeb_b200.observables import get_power_smoothed, power_Kaiser
    k, y = _outputs()
    for dlogk in (0.3, 1.359):
        got = get_power_smoothed(k=k, y=y, dlogk=dlogk, idx=4, param=PARAM)
        want = OB.get_power_smoothed(k, y, dlogk, 4, **PARAM)
        np.testing.assert_allclose(got, want, rtol=1e-12)
    got, _ = power_Kaiser(y=y, kmodes=k, bias=1.6, nmu=5, smooth_dlogk=1.359, param=PARAM)
    want, _ = OB.power_Kaiser(y, k, 1.6, 5, smooth_dlogk=1.359, **PARAM)
    np.testing.assert_allclose(got, want, rtol=1e-12)


@pytest.mark.parametrize("ell", [0, 1, 2, 4])
def test_gpu_xi_from_power_matches_oracle(torch_cuda, ell):
    from discoeb_b200.observables import get_xi_from_P
    k = np.geomspace(1e-4, 1e2, 2048)
    Pk = 2e4 * (k / 0.02) / (1 + (k / 0.02) ** 2.6) * np.exp(-(k / 5.0) ** 2)
    xi, r = get_xi_from_P(k=k, Pk=Pk, N=len(k), ell=ell)
    xi_ref, r_ref = OB.get_xi_from_P(k, Pk, ell=ell)
    np.testing.assert_allclose(r, r_ref, rtol=1e-15)
    np.testing.assert_allclose(xi, xi_ref, rtol=0, atol=1e-11 * max(np.abs(xi_ref).max(), 1e-300))
    # torch in, torch out, on the device
    torch = torch_cuda
    xt, rt = get_xi_from_P(k=torch.tensor(k, device="cuda"), Pk=torch.tensor(Pk, device="cuda"), ell=ell)
    assert xt.is_cuda and torch.equal(xt.cpu(), torch.tensor(xi))


def test_gpu_xi_rejects_odd_length(torch_cuda):
    from discoeb_b200.observables import get_xi_from_P
    with pytest.raises(ValueError):
        get_xi_from_P(k=np.geomspace(1e-3, 1.0, 7), Pk=np.ones(7))
