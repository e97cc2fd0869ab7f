"""CMB sources, line-of-sight multipoles and C_l on the GPU (discoeb_sources / discoeb_los /
discoeb_cell through discoeb_b200.cmb) against the CPU restatement on identical inputs."""
import os
import warnings

import numpy as np
import pytest

from conftest import GOLDEN, background
from oracle import cmb_oracle as C
from oracle import pyoracle as O

pytestmark = pytest.mark.gpu

L11 = dict(lmaxg=11, lmaxgp=11, lmaxr=11, lmaxnu=8, nqmax=3)


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("no CUDA device: the -m gpu tests need a GPU")
    return torch


@pytest.fixture(scope="module")
def gpu_states(torch_cuda):
    """Full RSA-projected states of 16 modes at the 320 CMB output times, from discoeb_fwd."""
    from discoeb_b200.cmb import cmb_aexp_out
    from discoeb_b200.perturbations import solve_modes
    bg = background("disco_notebook", 1024)
    a = cmb_aexp_out()
    tau = bg["tau_of_a_spline"].evaluate(a)
    ks = np.geomspace(1e-4, 0.5, 16)
    y = solve_modes(param=bg, kmodes=ks, tau_out=tau, rtol=1e-4, atol=1e-4, pcoeff=0.25, icoeff=0.8, dcoeff=0.0,
                    factormax=20.0, factormin=0.3, max_steps=4096, return_full=True, as_tensor=True, **L11)
    return bg, a, tau, ks, y


@pytest.fixture(params=["int8", "fp64"])
def contraction(request, torch_cuda):
    """the line of sight's frequency sum on the int8 tensor cores (default, 7 digit planes) or as an
    FP64 DGEMM; restored to the default afterwards"""
    from discoeb_b200.cmb import get_los_contraction, set_los_contraction
    before = get_los_contraction()
    set_los_contraction(request.param, 7)
    yield request.param
    set_los_contraction(*before)


def _close(got, want, rel):
    """Per mode (row), within rel of the row's largest magnitude."""
    scale = np.abs(want).max(axis=-1, keepdims=True) + 1e-300
    assert np.all(np.abs(got - want) <= rel * scale), float((np.abs(got - want) / scale).max())


def test_gpu_sources_match_oracle(gpu_states):
    from discoeb_b200.background import get_neutrino_momentum_bins
    from discoeb_b200.cmb import compute_sources
    bg, a, tau, ks, y = gpu_states
    src = compute_sources(param=bg, yout=y, kmodes=ks, aexp_out=a, **L11)
    yh = y.cpu().numpy()
    OP = O.OracleProblem(bg, de_guard_eps=1e-9, **L11)
    yp = np.stack([np.stack([OP.rhs(tau[j], yh[i, j], k) for j in range(len(tau))]) for i, k in enumerate(ks)])
    q, w = get_neutrino_momentum_bins(3)
    R = C.sources(yh, yp, ks, a, tau, bg, q, w, 11, 11, 11)
    want = {"S": R["S"], "S1": R["S1"], "S2": R["S2"], "S3": R["S3"], "S4": R["S4"],
            "alpha": R["metric"]["alpha"], "alphaprime": R["metric"]["alphaprime"],
            "alphapprime": R["metric"]["alphapprime"], "hprime": R["metric"]["hprime"],
            "polarization_term": R["pol"]["polarization_term"],
            "polarization_termpprime": R["pol"]["polarization_termpprime"],
            "drhonu": R["nu"]["drhonu"], "shear_nu_prime": R["nu"]["shear_nu_prime"], "E": R["E"]}
    for name, ref in want.items():
        _close(src[name].cpu().numpy(), ref, 1e-9)


@pytest.mark.parametrize("n_k_dense", [0, 200])
def test_gpu_theta_ell_and_cell_match_oracle(gpu_states, n_k_dense, contraction):
    from discoeb_b200.cmb import compute_Cell, compute_sources, compute_theta_ell
    bg, a, tau, ks, y = gpu_states
    S = compute_sources(param=bg, yout=y, kmodes=ks, aexp_out=a, **L11)["S"]
    tau0 = float(bg["tau_of_a_spline"].evaluate(1.0))
    th, kk = compute_theta_ell(300, ks, tau, S, tau0, n_fftlog=4096, n_k_dense=n_k_dense)
    th_o, kk_o = C.theta_ell(300, ks, tau, S.cpu().numpy(), tau0, n_fftlog=4096, n_k_dense=n_k_dense)
    np.testing.assert_allclose(kk.cpu().numpy(), kk_o, rtol=1e-14)
    _close(th.cpu().numpy(), th_o, 1e-9)
    cl = compute_Cell(th, kk, bg["n_s"], bg["k_p"]).cpu().numpy()
    np.testing.assert_allclose(cl, C.Cell(th.cpu().numpy(), kk_o, bg["n_s"], bg["k_p"]), rtol=1e-12)


@pytest.mark.parametrize("n_k_dense", [0, 200])
def test_gpu_e_mode_theta_ell_and_cross_cell_match_oracle(gpu_states, n_k_dense, contraction):
    from discoeb_b200.cmb import compute_Cell, compute_sources, compute_theta_ell
    bg, a, tau, ks, y = gpu_states
    src = compute_sources(param=bg, yout=y, kmodes=ks, aexp_out=a, **L11)
    tau0 = float(bg["tau_of_a_spline"].evaluate(1.0))
    th, kk = compute_theta_ell(300, ks, tau, src["S"], tau0, n_fftlog=4096, n_k_dense=n_k_dense)
    the, kk2 = compute_theta_ell(300, ks, tau, src["E"], tau0, n_fftlog=4096, n_k_dense=n_k_dense, kind="E")
    the_o, kk_o, mag = C.theta_ell_E(300, ks, tau, src["E"].cpu().numpy(), tau0, n_fftlog=4096,
                                     n_k_dense=n_k_dense, abs_sums=True)
    np.testing.assert_allclose(kk2.cpu().numpy(), kk_o, rtol=1e-14)
    # 1e-9 of each mode's largest multipole, plus the rounding scale of the FFTLog sums: at high k
    # the recurrence's three terms cancel by ~(k chi)^2 near l = 8, where eps times the sum of
    # magnitudes reaches ~5e-9 of the row's largest value on the dense k grid (the int8 contraction
    # with 7 digit planes uses 0.35 of this bound there, the FP64 one 0.20)
    got = the.cpu().numpy()
    bound = 1e-9 * np.abs(the_o).max(axis=-1, keepdims=True) + 32 * np.finfo(float).eps * mag
    assert np.all(np.abs(got - the_o) <= bound), float((np.abs(got - the_o) / bound).max())
    cte = compute_Cell(th, kk, bg["n_s"], bg["k_p"], theta_ell_b=the).cpu().numpy()
    ref = C.Cell(th.cpu().numpy(), kk_o, bg["n_s"], bg["k_p"], the.cpu().numpy())
    np.testing.assert_allclose(cte, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())


def test_gpu_cmb_spectrum_pipeline(torch_cuda):
    """compute_Cell_spectrum_from_cosmo_params at the reference's defaults: every stage on the
    GPU equals the restated chain applied to the GPU's own states, and D_l is within the
    reference test's bound of CAMB (mean relative error < 1%)."""
    from discoeb_b200.background import get_neutrino_momentum_bins
    from discoeb_b200.cmb import compute_Cell_spectrum_from_cosmo_params, compute_Dell
    p = {"Omegam": 0.3099, "Omegab": 0.0488911, "H0": 67.742, "n_s": 0.96822, "A_s": 2.1064e-09, "mnu": 0.06,
         "Tcmb": 2.7255, "YHe": 0.248, "Neff": 2.046, "Nmnu": 1, "w_DE_0": -0.99, "w_DE_a": 0.0, "cs2_DE": 1.0,
         "Omegak": 0.0, "k_p": 0.05}
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        cells, param, mid = compute_Cell_spectrum_from_cosmo_params(p, return_intermediates=True,
                                                                    spectra=("TT", "TE", "EE"))
    cell = cells["TT"]
    ell, D = compute_Dell(cell, param["A_s"], param["Tcmb"])
    g = np.load(os.path.join(GOLDEN, "reference_cmb_golden.npz"))
    Dc = np.interp(ell, g["camb:ell"], g["camb:D_ell"])
    assert np.mean(np.abs(D - Dc) / Dc) < 0.01
    # the same chain restated on the CPU from the GPU's states
    yh = mid["y"].cpu().numpy()
    ks, a, tau = mid["kmodes"], mid["aexp_out"], mid["tau"]
    OP = O.OracleProblem(param, de_guard_eps=1e-9, **L11)
    yp = np.stack([np.stack([OP.rhs(tau[j], yh[i, j], k) for j in range(len(tau))]) for i, k in enumerate(ks)])
    q, w = get_neutrino_momentum_bins(3)
    R = C.sources(yh, yp, ks, a, tau, param, q, w, 11, 11, 11)
    th, kk = C.theta_ell(2500, ks, tau, R["S"], float(param["tau_of_a_spline"].evaluate(1.0)), 16384, 8192)
    cl_o = C.Cell(th, kk, param["n_s"], param["k_p"])
    np.testing.assert_allclose(cell[2:], cl_o[2:], rtol=1e-8)
    # E-mode polarisation: the restated chain, and the CLASS EE / TE the reference commits (no
    # reionisation) at the level the reference holds TT against CLASS and CAMB
    tau0 = float(param["tau_of_a_spline"].evaluate(1.0))
    the, _ = C.theta_ell_E(2500, ks, tau, R["E"], tau0, 16384, 8192)
    ee_o = C.Cell(the, kk, param["n_s"], param["k_p"])
    te_o = C.Cell(th, kk, param["n_s"], param["k_p"], the)
    np.testing.assert_allclose(cells["EE"][2:], ee_o[2:], rtol=1e-7)
    sc = np.sqrt(np.abs(cl_o[2:] * ee_o[2:]))
    assert np.all(np.abs(cells["TE"][2:] - te_o[2:]) <= 1e-7 * sc)
    cls = {f: np.interp(ell, g["class:ell"], g[f"class:D_ell_{f}"]) for f in ("TT", "EE", "TE")}
    _, DEE = compute_Dell(cells["EE"], param["A_s"], param["Tcmb"])
    _, DTE = compute_Dell(cells["TE"], param["A_s"], param["Tcmb"])
    ree = np.abs(DEE / cls["EE"] - 1)
    rte = np.abs(DTE - cls["TE"]) / np.sqrt(cls["TT"] * cls["EE"])
    assert ree.mean() < 0.02 and np.median(ree) < 0.015, (ree.mean(), np.median(ree))
    assert rte.mean() < 0.01, rte.mean()


def test_gpu_fused_solve_and_sources_equal_the_two_stages(gpu_states):
    """discoeb_fwd_sources (the solve with the source assembly in its output stage) against
    discoeb_fwd + discoeb_sources on the same modes: the same states and fields to rounding (the
    same source code, compiled into two kernels: measured 3.5e-11 on the states), and the
    pipeline's C_l with fused_sources equal to the two-stage one."""
    import warnings
    from discoeb_b200.cmb import compute_Cell_spectrum_from_cosmo_params, compute_sources, solve_sources
    bg, a, tau, ks, y = gpu_states
    src = compute_sources(param=bg, yout=y, kmodes=ks, aexp_out=a, **L11)
    for _ in range(2):
        fused, yf = solve_sources(param=bg, kmodes=ks, aexp_out=a, rtol=1e-4, atol=1e-4, max_steps=4096,
                                  return_states=True, **L11)
        _close(yf.cpu().numpy(), y.cpu().numpy(), 1e-9)
        for name in src:
            _close(fused[name].cpu().numpy(), src[name].cpu().numpy(), 1e-9)
    p = {"Omegam": 0.3099, "Omegab": 0.0488911, "H0": 67.742, "n_s": 0.96822, "A_s": 2.1064e-09, "mnu": 0.06,
         "Tcmb": 2.7255, "YHe": 0.248, "Neff": 2.046, "Nmnu": 1, "w_DE_0": -0.99, "w_DE_a": 0.0, "cs2_DE": 1.0,
         "Omegak": 0.0, "k_p": 0.05}
    opts = dict(ellmax=600, nmodes=32, n_k_dense=1024, n_fftlog=4096, spectra=("TT", "EE"))
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        c1, _ = compute_Cell_spectrum_from_cosmo_params(p, **opts)
        c2, _ = compute_Cell_spectrum_from_cosmo_params(p, fused_sources=True, **opts)
    for name in opts["spectra"]:
        np.testing.assert_allclose(c2[name][2:], c1[name][2:], rtol=1e-8, atol=0)
