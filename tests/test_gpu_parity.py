"""GPU solver against the oracle (run on a B200 with -m gpu).  Every call goes through the
C ABI of libdiscoeb_b200.so (discoeb_fwd / discoeb_rhs)."""
import numpy as np
import pytest

from conftest import background
from oracle import pyoracle as O

pytestmark = pytest.mark.gpu

L143 = dict(lmaxg=12, lmaxgp=12, lmaxr=17, lmaxnu=17, nqmax=5)
L65 = dict(lmaxg=12, lmaxgp=12, lmaxr=17, lmaxnu=3, nqmax=3)
A4 = np.array([1 / 3, 0.5, 2 / 3, 1.0])


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("no CUDA device: the -m gpu tests need a GPU")
    return torch


def test_gpu_rhs_matches_oracle(torch_cuda):
    from discoeb_b200.perturbations import compute_time_derivatives
    bg = background("lcdm_mnu", 256)
    OP = O.OracleProblem(bg, de_guard_eps=1e-9, **L143)
    rng = np.random.default_rng(0)
    ks = np.array([1e-4, 1e-2, 0.3, 5.0])
    tau = bg["tau_of_a_spline"].evaluate(np.array([1e-4, 1e-3, 0.05, 0.7]))
    y = np.zeros((4, 4, OP.n))
    for i, k in enumerate(ks):
        ts = 0.99 * OP.start_time(k)
        ys, _ = OP.solve([k], ts, OP.ics(ts, k), tau, rtol=1e-6, atol=1e-9, max_steps=100000)
        y[i] = ys[0] * (1 + 0.01 * rng.standard_normal(ys[0].shape))
    f = compute_time_derivatives(y, tau, ks, bg, **L143)
    for i, k in enumerate(ks):
        for j, t in enumerate(tau):
            fo = OP.rhs(t, y[i, j], k)
            np.testing.assert_allclose(f[i, j], fo, rtol=0, atol=1e-12 * np.abs(fo).max())


def _oracle_outputs(bg, ks, aout, L, rtol, atol, guard=1e-9, full=False):
    y, _, st = O.evolve_perturbations(param=bg, aexp_out=aout, kmin=0, kmax=0, num_k=0, rtol=rtol, atol=atol,
                                      max_steps=200000, kmodes=ks, mode="clip", de_guard_eps=guard, return_full=full,
                                      **L)
    assert all(s[3] == 0 for s in st)
    return y


def test_gpu_forward_matches_oracle_same_algorithm(torch_cuda):
    # same method, controller and step clipping as the oracle's clip mode: the step sequences
    # coincide, so the results agree far below the tolerance
    from discoeb_b200.perturbations import solve_modes
    bg = background("lcdm_mnu", 256)
    ks = np.geomspace(1e-4, 10.0, 12)
    tout = bg["tau_of_a_spline"].evaluate(A4)
    y, status, nsteps = solve_modes(param=bg, kmodes=ks, tau_out=tout, rtol=1e-5, atol=1e-8, pcoeff=0.25, icoeff=0.8,
                                    dcoeff=0.0, factormax=20.0, factormin=0.3, max_steps=4096, return_full=False,
                                    return_stats=True, **L143)
    assert (status == 0).all()
    yo = _oracle_outputs(bg, ks, A4, L143, 1e-5, 1e-8)
    for idx in (0, 2, 4, 6, 8, 10):
        np.testing.assert_allclose(y[:, :, idx], yo[:, :, idx], rtol=1e-6, atol=1e-12)


@pytest.mark.parametrize("name", ["lcdm_massless", "lcdm_mnu"])
def test_gpu_pk_within_1em4_of_converged_oracle(torch_cuda, name):
    from discoeb_b200.perturbations import evolve_perturbations, get_power
    L = L65 if name == "lcdm_massless" else L143
    kmax = 1.0 if name == "lcdm_massless" else 10.0
    aout = np.array([1.0]) if name == "lcdm_massless" else A4
    bg = background(name, 256)
    y, k, _ = evolve_perturbations(param=dict(bg), aexp_out=aout, kmin=1e-4, kmax=kmax, num_k=16, rtol=1e-5,
                                   atol=1e-8, k_sampling_method="log", max_steps=4096, **L)
    yo = _oracle_outputs(bg, k, aout, L, 1e-10, 1e-13)
    P = get_power(k=k[:, None], y=y, idx=4, param=bg)
    Po = get_power(k=k[:, None], y=yo, idx=4, param=bg)
    rel = np.abs(P / Po - 1)
    assert rel.max() < 1e-4, rel.max()


def test_gpu_full_state_and_projection(torch_cuda):
    from discoeb_b200.perturbations import evolve_perturbations
    bg = background("disco_notebook", 1024)
    aout = np.geomspace(1e-3, 1.0, 7)
    y, k, p = evolve_perturbations(param=dict(bg), aexp_out=aout, kmin=1e-3, kmax=1.0, num_k=6, rtol=1e-5, atol=1e-8,
                                   return_full=True, k_sampling_method="log", max_steps=4096)
    assert y.shape == (6, 7, 72) and p["nout"] == 7
    yo = _oracle_outputs(bg, k, aout, dict(lmaxg=11, lmaxgp=11, lmaxr=11, lmaxnu=8, nqmax=3), 1e-5, 1e-8, 0.0,
                         full=True)
    np.testing.assert_allclose(y[:, :, 3], yo[:, :, 3], rtol=2e-5)  # same algorithm; rare accept flips
    np.testing.assert_allclose(y[:, :, 7], yo[:, :, 7], rtol=3e-5, atol=1e-9 * np.abs(yo[:, :, 7]).max())


def test_gpu_edge_cases(torch_cuda):
    from discoeb_b200.perturbations import evolve_perturbations, solve_modes
    bg = background("lcdm_massless", 256)
    kw = dict(rtol=1e-5, atol=1e-8, pcoeff=0.25, icoeff=0.8, dcoeff=0.0, factormax=20.0, factormin=0.3,
              return_full=False, **L65)
    tout = bg["tau_of_a_spline"].evaluate(np.array([1.0]))
    y = solve_modes(param=bg, kmodes=np.zeros(0), tau_out=tout, max_steps=100, **kw)
    assert y.shape == (0, 1, 20)
    with pytest.raises(RuntimeError, match="max_steps"):
        solve_modes(param=bg, kmodes=np.array([0.1]), tau_out=tout, max_steps=3, **kw)
    y, status, nsteps = solve_modes(param=bg, kmodes=np.array([0.1, 0.01]), tau_out=tout, max_steps=3,
                                    on_failure="ignore", return_stats=True, **kw)
    assert (status == 1).all() and (nsteps == 3).all() and np.isnan(y).all()
    with pytest.raises(ValueError):
        solve_modes(param=bg, kmodes=np.array([0.1]), tau_out=np.array([100.0, 50.0]), max_steps=100, **kw)
    with pytest.raises(NotImplementedError):
        evolve_perturbations(param=dict(bg, use_tca=True), aexp_out=[1.0], kmin=1e-3, kmax=1.0, num_k=2, **L65)


def test_gpu_full_size_properties(torch_cuda):
    # the 512-mode, 4-redshift massive-neutrino problem: all modes finish, results are
    # bitwise reproducible, and P(k) scales between redshifts like the linear growth
    from discoeb_b200.perturbations import evolve_perturbations, get_power
    from discoeb_b200.workloads import workload
    w = workload("pk_lcdm_mnu_k512_z4")
    bg = background("lcdm_mnu", 256)
    kw = {k: w[k] for k in ("kmin", "kmax", "num_k", "aexp_out", "rtol", "atol", "lmaxg", "lmaxgp", "lmaxr", "lmaxnu",
                            "nqmax")}
    y1, k, _ = evolve_perturbations(param=dict(bg), k_sampling_method="log", max_steps=4096, **kw)
    y2, _, _ = evolve_perturbations(param=dict(bg), k_sampling_method="log", max_steps=4096, **kw)
    assert np.array_equal(y1, y2)
    P = get_power(k=k[:, None], y=y1, idx=4, param=bg)
    assert np.isfinite(P).all() and (P > 0).all()
    g2 = P[:, 0] / P[:, -1]  # z = 2 over z = 0
    assert (g2 < 1).all() and (g2 > 0.05).all()
    assert np.ptp(g2[k < 1e-2]) < 0.02  # scale-independent growth on large scales
