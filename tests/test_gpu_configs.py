"""The GPU solver against the converged oracle at the sizes of the benchmark configurations:

* the batched massive-neutrino configuration (l_max 12/12/17/17, 5 momentum bins, 143 variables):
  64 modes over [1e-4, 10] /Mpc at z = 2, 1, 0.5, 0;
* the uneven batch: 8 draws of the seeded cosmology box (numpy default_rng(0)), 4 of them with
  w(a) crossing -1, in one multi-cosmology launch (the crossing draws have no converged value: the
  fluid equations are singular at the crossing; see the test);
* the CMB configuration's solver size (photon and polarisation l_max 50, 219 variables) on a few
  modes and output times;
* the gradient kernel against the same tangent code compiled for one host thread
  (tests/cpu_model), mode by mode.

The oracle runs the same equations at rtol 1e-10 / atol 1e-13 with steps ending on the output
times; the bar is the benchmark's 1e-4 relative error.
"""
import ctypes
import warnings

import numpy as np
import pytest

from conftest import background
from oracle import pyoracle as O

pytestmark = pytest.mark.gpu

L143 = dict(lmaxg=12, lmaxgp=12, lmaxr=17, lmaxnu=17, nqmax=5)
L219 = dict(lmaxg=50, lmaxgp=50, lmaxr=17, lmaxnu=17, nqmax=5)
A4 = np.array([1 / 3, 0.5, 2 / 3, 1.0])
TIGHT = dict(rtol=1e-10, atol=1e-13)


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("no CUDA device: the -m gpu tests need a GPU")
    return torch


def _oracle(bg, ks, aout, L, full=False):
    y, _, st = O.evolve_perturbations(param=bg, aexp_out=aout, kmin=0, kmax=0, num_k=0, max_steps=400000, kmodes=ks,
                                      mode="clip", de_guard_eps=1e-9, return_full=full, **TIGHT, **L)
    assert all(s[3] == 0 for s in st), st
    return y


def test_gpu_pk_64_modes_four_redshifts_within_1em4(torch_cuda):
    from discoeb_b200.perturbations import evolve_perturbations, get_power
    bg = background("lcdm_mnu", 256)
    y, k, _ = evolve_perturbations(param=dict(bg), aexp_out=A4, kmin=1e-4, kmax=10.0, num_k=64, rtol=1e-5, atol=1e-8,
                                   k_sampling_method="log", max_steps=100000, **L143)
    yo = _oracle(bg, k, A4, L143)
    P = get_power(k=k[:, None], y=y, idx=4, param=bg)
    Po = get_power(k=k[:, None], y=yo, idx=4, param=bg)
    rel = np.abs(P / Po - 1)
    assert rel.shape == (64, 4)
    assert rel.max() < 1e-4, (rel.max(), np.unravel_index(rel.argmax(), rel.shape))


def test_gpu_uneven_batch_draws_with_phantom_crossing_within_1em4(torch_cuda):
    from discoeb_b200.background import evolve_background
    from discoeb_b200.gradients import theta_to_params
    from discoeb_b200.perturbations import get_power, solve_cosmologies
    from discoeb_b200.workloads import crosses_phantom_divide, sample_thetas
    thetas = sample_thetas(1024, seed=0)
    cross = [t for t in thetas if crosses_phantom_divide(t)][:4]
    plain = [t for t in thetas if not crosses_phantom_divide(t)][:4]
    draws = cross + plain
    assert len(cross) == 4
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        bgs = [evolve_background(param=theta_to_params(t)) for t in draws]
    ks = np.geomspace(1e-4, 5.0, 12)
    aout = np.array([1.0])
    y, status, _ = solve_cosmologies(params=bgs, kmodes=ks, aexp_out=aout, rtol=1e-5, atol=1e-8, max_steps=100000,
                                     return_stats=True, **L143)
    assert (status == 0).all()
    worst = []
    for c, bg in enumerate(bgs[4:]):
        yo = _oracle(bg, ks, aout, L143)
        P = get_power(k=ks[:, None], y=y[4 + c], idx=4, param=bg)
        Po = get_power(k=ks[:, None], y=yo, idx=4, param=bg)
        worst.append(float(np.abs(P / Po - 1).max()))
    assert max(worst) < 1e-4, worst
    # where w(a) crosses -1 the reference's fluid equations are singular (cs2 k^2 delta_q / (1 + w),
    # perturbations.py:518-523) and the solution depends on how the steps straddle the crossing:
    # the CPU restatement itself moves by ~1e-2 between rtol 1e-5 and 1e-11 on these draws, so no
    # converged value exists to compare with; the GPU solves them (every mode succeeds, finite P)
    assert np.isfinite(y[:4]).all()


def test_gpu_cmb_size_solver_within_1em4(torch_cuda):
    # 219 variables (photon and polarisation hierarchies to l = 50): whole states at six output
    # times spanning recombination to today, and P(k) today
    from discoeb_b200.perturbations import evolve_perturbations, get_power
    bg = background("lcdm_mnu", 256)
    aout = np.array([7e-4, 1e-3, 2e-3, 0.01, 0.1, 1.0])
    y, k, _ = evolve_perturbations(param=dict(bg), aexp_out=aout, kmin=5e-5, kmax=0.5, num_k=5, rtol=1e-5, atol=1e-8,
                                   k_sampling_method="log", max_steps=100000, return_full=True, **L219)
    assert y.shape == (5, 6, 219)
    yo = _oracle(bg, k, aout, L219, full=True)
    for idx in (2, 3, 5, 6, 7):  # eta, delta_c, delta_b, theta_b, delta_gamma
        scale = np.abs(yo[:, :, idx]).max(axis=1, keepdims=True)
        err = np.abs(y[:, :, idx] - yo[:, :, idx]) / scale
        assert err.max() < 1e-4, (idx, err.max())
    yf, _, _ = evolve_perturbations(param=dict(bg), aexp_out=[1.0], kmin=5e-5, kmax=0.5, num_k=5, rtol=1e-5,
                                    atol=1e-8, k_sampling_method="log", max_steps=100000, **L219)
    yfo = _oracle(bg, k, [1.0], L219)
    P = get_power(k=k[:, None], y=yf, idx=4, param=bg)
    Po = get_power(k=k[:, None], y=yfo, idx=4, param=bg)
    assert np.abs(P / Po - 1).max() < 1e-4


def test_gpu_jacobian_equals_cpu_build_of_the_tangent_code(torch_cuda, shim):
    """discoeb_jvp's output-field tangents against stepper.cuh / model.cuh compiled for one host
    thread (the same arithmetic; separately compiled code can flip a step acceptance, which moves
    a result by up to the solver tolerance, so the bar is 1e-6 of each direction's scale)."""
    from discoeb_b200 import _abi
    from discoeb_b200.gradients import JacobianProblem, cosmology_prologue
    theta = dict(omega_c=0.120, omega_b=0.0224, h=0.674, n_s=0.965, ln10As=np.log(21.0), w0=-0.9, wa=0.1,
                 m_nu=0.06)
    ks = np.geomspace(1e-3, 1.0, 6)
    aout = np.array([0.5, 1.0])
    prob = JacobianProblem(theta, aexp_out=aout, kmodes=ks, rtol=1e-5, atol=1e-8, **L143)
    prob.launch()
    inv = prob.inv
    yd_gpu = prob.d_outd.cpu().numpy()[:, inv]  # [dir, K, nout, 20]
    y_gpu = prob.d_out.cpu().numpy()[inv]
    pro = cosmology_prologue(theta, aout, ks, L143)
    bg, tau_out, tau_start, y0, sw, tans = (pro[k] for k in ("bg", "tau_out", "tau_start", "y0", "sw", "tans"))
    keep = []
    C = _abi.make_cosmo(bg, de_guard_eps=1e-9, table_ptrs=_abi.host_table_ptrs(bg, keep), **L143)
    ctrl = _abi.DiscoebControl(1e-5, 1e-8, 0.25, 0.8, 0.0, 20.0, 0.3, 100000, 0, 0, 0)
    n = prob.n
    dp = ctypes.POINTER(ctypes.c_double)
    p = lambda a: np.ascontiguousarray(a).ctypes.data_as(dp)  # noqa: E731
    for d, tan in enumerate(tans):
        tn = _abi.DiscoebTangent()
        for f, v in tan["scalars"].items():
            setattr(tn, f, v)
        for short, (yy, SS) in tan["tables"].items():
            yy, SS = np.ascontiguousarray(yy), np.ascontiguousarray(SS)
            keep += [yy, SS]
            setattr(tn, short + "_y", yy.ctypes.data)
            setattr(tn, short + "_S", SS.ctypes.data)
        for i, k in enumerate(ks):
            yo, ydo = np.zeros((2, n)), np.zeros((2, n))
            stats = (ctypes.c_int * 3)()
            y0i, yd0i = np.ascontiguousarray(y0[i]), np.ascontiguousarray(tan["y0"][i])
            shim.shim_solve_mode_tangent(ctypes.byref(C), ctypes.byref(tn), ctypes.byref(ctrl), k, tau_start[i],
                                         p(y0i), p(yd0i), p(sw[i]), 2, p(tau_out), p(yo), p(ydo), stats, None, 0)
            assert stats[0] == 0
            for j in range(2):
                f, col0 = np.zeros(n), np.zeros(n)
                shim.shim_rhs(ctypes.byref(C), tau_out[j], p(yo[j]), k, -1, p(f), p(col0))
                ydm = ydo[j] + f * tan["tau_out"][j]  # the state's tangent at the moving output time
                o, od = np.zeros(20), np.zeros(20)
                shim.shim_projected_output_tangent(ctypes.byref(C), ctypes.byref(tn), k, tau_out[j], p(yo[j]),
                                                   p(ydm), p(o), p(od))
                np.testing.assert_allclose(o[4], y_gpu[i, j, 4], rtol=1e-6)
                scale = np.abs(yd_gpu[d, :, j, 4]).max()
                assert abs(od[4] - yd_gpu[d, i, j, 4]) <= 1e-6 * scale, (d, i, j, od[4], yd_gpu[d, i, j, 4])


def test_gpu_mixed_precision_forward_within_1em4(torch_cuda):
    """The mixed-precision form (FP32 chain factors, one FP64 refinement of every chain solve) on
    the batched massive-neutrino configuration: within the benchmark's 1e-4 of the converged oracle
    and within the solver tolerance of the FP64 form."""
    from discoeb_b200.perturbations import get_power, solve_modes
    bg = background("lcdm_mnu", 256)
    ks = np.geomspace(1e-4, 10.0, 16)
    tout = bg["tau_of_a_spline"].evaluate(A4)
    common = dict(param=dict(bg), kmodes=ks, tau_out=tout, rtol=1e-5, atol=1e-8, pcoeff=0.25, icoeff=0.8,
                  dcoeff=0.0, factormax=20.0, factormin=0.3, max_steps=100000, return_full=False, return_stats=True,
                  **L143)
    ym, st_m, n_m = solve_modes(method="structured-mixed", **common)
    yd, st_d, n_d = solve_modes(method="structured", **common)
    assert (st_m == 0).all() and (st_d == 0).all()
    # the refined solves round differently, which moves the error control's step choices: on one
    # high-k mode the measured step count differed by 3.6%
    assert np.all(np.abs(n_m - n_d) <= np.maximum(2, 0.05 * n_d)), (n_m, n_d)
    Pm = get_power(k=ks[:, None], y=ym, idx=4, param=bg)
    Pd = get_power(k=ks[:, None], y=yd, idx=4, param=bg)
    Po = get_power(k=ks[:, None], y=_oracle(bg, ks, A4, L143), idx=4, param=bg)
    assert np.abs(Pm / Po - 1).max() < 1e-4
    assert np.abs(Pm / Pd - 1).max() < 1e-5
