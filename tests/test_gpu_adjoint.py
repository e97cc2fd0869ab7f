"""The discrete adjoint on the GPU (discoeb_fwd_record + discoeb_bwd + discoeb_bwd_contract,
through gradients.AdjointProblem / AdjointBatch): its gradient of a scalar loss equals the
forward-mode Jacobian contracted with the loss weights, and central differences of the whole
pipeline."""
import math
import warnings

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

L143 = dict(lmaxg=12, lmaxgp=12, lmaxr=17, lmaxnu=17, nqmax=5)
L65 = dict(lmaxg=12, lmaxgp=12, lmaxr=17, lmaxnu=3, nqmax=3)
A4 = np.array([1 / 3, 0.5, 2 / 3, 1.0])
THETA = dict(omega_c=0.120, omega_b=0.0224, h=0.674, n_s=0.965, ln10As=math.log(21.0), w0=-0.9, wa=0.1, m_nu=0.06)


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("no CUDA device: the -m gpu tests need a GPU")
    return torch


@pytest.mark.parametrize("every", [1, 16])
def test_gpu_adjoint_equals_contracted_forward_jacobian(torch_cuda, every):
    from discoeb_b200.gradients import AdjointProblem, JacobianProblem
    kw = dict(aexp_out=A4, kmin=1e-4, kmax=10.0, num_k=16, rtol=1e-5, atol=1e-8, **L143)
    jp = JacobianProblem(THETA, **kw)
    jp.launch()
    P, J, status, _ = jp.result()
    w = np.random.default_rng(0).uniform(0.5, 2.0, P.shape) / P
    ap = AdjointProblem(THETA, checkpoint_every=every, **kw)
    ap.launch_forward()
    Pa, sa, _ = ap.forward_power()
    assert (sa == 0).all()
    np.testing.assert_allclose(Pa[0], P, rtol=2e-5)  # separately compiled kernels: rare accept flips
    ap.launch_backward(w)
    g = ap.gradient(w)[0]
    expect = np.einsum("dkn,kn->d", J, w)
    np.testing.assert_allclose(g, expect, rtol=1e-8, atol=1e-12 * np.abs(expect).max())


def test_gpu_adjoint_jacobian_rows_equal_forward_jacobian(torch_cuda):
    # one reverse sweep per mode with that mode's P(k, z = 0) as the cotangent: the whole
    # Jacobian dP(k, z=0)/dtheta (the gradient configuration) row by row
    from discoeb_b200.gradients import AdjointProblem, JacobianProblem
    kw = dict(aexp_out=A4, kmin=1e-4, kmax=10.0, num_k=24, rtol=1e-5, atol=1e-8, **L143)
    jp = JacobianProblem(THETA, **kw)
    jp.launch()
    P, J, _, _ = jp.result()
    ap = AdjointProblem(THETA, **kw)
    ap.launch_forward()
    ap.launch_jacobian_rows(out_index=-1)
    Ja = ap.jacobian_rows()[0]
    scale = np.abs(J[:, :, -1]).max(axis=1, keepdims=True)
    assert np.all(np.abs(Ja - J[:, :, -1]) <= 1e-8 * scale), float((np.abs(Ja - J[:, :, -1]) / scale).max())


def test_gpu_adjoint_matches_central_differences(torch_cuda):
    """dL/dtheta of L = sum w P against central differences of step 1e-4 |theta_i| of the whole
    pipeline at rtol 1e-10, with the start times, switch times and Recfast steps held at the base
    point (the derivative forward-mode AD through the reference defines)."""
    from discoeb_b200.background import evolve_background
    from discoeb_b200.gradients import THETA_NAMES, AdjointProblem, theta_to_params
    from discoeb_b200.perturbations import (approximation_switch_times, determine_starting_time, get_power,
                                            solve_modes)
    solver = dict(rtol=1e-10, atol=1e-13, max_steps=400000)
    aout = (0.5, 1.0)
    ap = AdjointProblem(THETA, aexp_out=aout, kmin=1e-3, kmax=0.5, num_k=8, step_capacity=65536, **solver, **L143)
    ap.launch_forward()
    P = ap.forward_power()[0][0]
    k = ap.kmodes
    w = np.random.default_rng(1).uniform(0.5, 2.0, P.shape) / P
    ap.launch_backward(w)
    g = ap.gradient(w)[0]

    def power(theta, trace=None, replay=None, **fixed):
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")
            bg = evolve_background(param=theta_to_params(theta), trace=trace, replay=replay)
        tout = bg["tau_of_a_spline"].evaluate(np.asarray(aout))
        y = solve_modes(param=bg, kmodes=k, tau_out=tout, pcoeff=0.25, icoeff=0.8, dcoeff=0.0, factormax=20.0,
                        factormin=0.3, return_full=False, **fixed, **solver, **L143)
        return get_power(k=k[:, None], y=y, idx=4, param=bg), bg

    trace = {}
    P0, bg = power(THETA, trace=trace)
    tout = bg["tau_of_a_spline"].evaluate(np.asarray(aout))
    fixed = dict(tau_start=0.99 * np.minimum(tout.min(), determine_starting_time(param=bg, k=k)),
                 switch_tau=approximation_switch_times(bg, k))
    worst = {}
    for i, name in enumerate(THETA_NAMES):
        eps = 1e-4 * abs(THETA[name])
        tp, tm = dict(THETA), dict(THETA)
        tp[name] += eps
        tm[name] -= eps
        fd = (np.sum(w * power(tp, replay=trace, **fixed)[0]) - np.sum(w * power(tm, replay=trace, **fixed)[0])) \
            / (2 * eps)
        worst[name] = abs(g[i] - fd) / abs(fd)
    assert max(worst.values()) < 2e-4, worst


def test_gpu_adjoint_batch_equals_single_cosmology(torch_cuda):
    from discoeb_b200.gradients import AdjointBatch, AdjointProblem
    from discoeb_b200.workloads import sample_thetas
    thetas = sample_thetas(3, seed=4)
    ks = np.geomspace(1e-3, 1.0, 5)
    kw = dict(aexp_out=(0.5, 1.0), rtol=1e-5, atol=1e-8, **L65)
    batch = AdjointBatch(thetas, kmodes=ks, **kw)
    batch.launch_forward()
    P, status, _ = batch.forward_power()
    w = np.random.default_rng(2).uniform(0.5, 2.0, P.shape) / P
    batch.launch_backward(w)
    G = batch.gradient(w)
    for c, th in enumerate(thetas):
        one = AdjointProblem(th, kmodes=ks, **kw)
        one.launch_forward()
        P1 = one.forward_power()[0]
        np.testing.assert_array_equal(P1[0], P[c])
        one.launch_backward(w[c])
        np.testing.assert_allclose(one.gradient(w[c])[0], G[c], rtol=1e-11)  # atomics: equal to rounding


def test_gpu_adjoint_record_capacity_is_reported(torch_cuda):
    from discoeb_b200.gradients import AdjointProblem
    ap = AdjointProblem(THETA, aexp_out=(1.0,), kmin=1e-2, kmax=1.0, num_k=3, step_capacity=5, **L65)
    ap.launch_forward()
    _, status, _ = ap.forward_power(on_failure="ignore")
    assert (status == 7).all()  # DISCOEB_RECORD_FULL
    ap.launch_backward(np.ones((3, 1)))
    with pytest.raises(RuntimeError, match="record"):
        ap.gradient(np.ones((3, 1)))


def test_gpu_autograd_function_adjoint_equals_forward_mode(torch_cuda):
    torch = torch_cuda
    from discoeb_b200.gradients import THETA_NAMES, power_spectrum_function
    opts = dict(aexp_out=(1.0,), kmin=1e-3, kmax=0.3, num_k=6, **L143)
    theta0 = [THETA[n] for n in THETA_NAMES]
    grads = []
    for mode in ("forward", "adjoint"):
        PK = power_spectrum_function(gradient=mode, **opts)
        theta = torch.tensor(theta0, dtype=torch.float64, device="cuda", requires_grad=True)
        P = PK.apply(theta)
        wts = torch.linspace(0.5, 2.0, P.numel(), dtype=torch.float64, device="cuda").reshape(P.shape)
        (P * wts / P.detach()).sum().backward()
        grads.append(theta.grad.cpu().numpy())
    np.testing.assert_allclose(grads[1], grads[0], rtol=1e-8, atol=1e-12 * np.abs(grads[0]).max())
