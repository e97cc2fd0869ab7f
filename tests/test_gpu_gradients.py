"""Gradients of P(k) on the GPU (discoeb_jvp through gradients.JacobianProblem), against the
forward entry point and against central finite differences of the whole pipeline."""
import math
import warnings

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

L143 = dict(lmaxg=12, lmaxgp=12, lmaxr=17, lmaxnu=17, nqmax=5)
A4 = np.array([1 / 3, 0.5, 2 / 3, 1.0])
THETA = dict(omega_c=0.120, omega_b=0.0224, h=0.674, n_s=0.965, ln10As=math.log(21.0), w0=-0.9, wa=0.1, m_nu=0.06)


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("no CUDA device: the -m gpu tests need a GPU")
    return torch


def _power(theta, kmodes, aexp_out, trace=None, replay=None, **solver):
    """P(k) of the forward path (evolve_background + solve_modes + get_power), and the
    background."""
    from discoeb_b200.background import evolve_background
    from discoeb_b200.gradients import theta_to_params
    from discoeb_b200.perturbations import get_power, solve_modes
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        bg = evolve_background(param=theta_to_params(theta), trace=trace, replay=replay)
    tout = bg["tau_of_a_spline"].evaluate(np.asarray(aexp_out, dtype=np.float64))
    y = solve_modes(param=bg, kmodes=kmodes, tau_out=tout, pcoeff=0.25, icoeff=0.8, dcoeff=0.0, factormax=20.0,
                    factormin=0.3, return_full=False, **solver, **L143)
    return get_power(k=kmodes[:, None], y=y, idx=4, param=bg), bg


def test_gpu_jvp_values_match_forward_solve(torch_cuda):
    from discoeb_b200.gradients import JacobianProblem
    prob = JacobianProblem(THETA, aexp_out=A4, kmin=1e-4, kmax=10.0, num_k=24, rtol=1e-5, atol=1e-8, **L143)
    prob.launch()
    P, J, status, nsteps = prob.result()
    assert (status == 0).all()
    P_fwd, _ = _power(THETA, prob.kmodes, A4, rtol=1e-5, atol=1e-8, max_steps=100000)
    # same algorithm: the value part of the tangent solve is the forward solve.  The two kernels
    # are compiled separately (their fused multiply-adds may differ in the last bit), and the
    # step-size control can turn such a difference into a different accept decision, which moves
    # the result by up to the solver tolerance (rtol 1e-5)
    np.testing.assert_allclose(P, P_fwd, rtol=2e-5)
    assert np.isfinite(J).all()


def test_gpu_jacobian_matches_central_differences(torch_cuda):
    """dP/dtheta against central differences with relative step 1e-4.

    The perturbation solves run at rtol 1e-10 so that the difference quotient of the adaptive
    solve (which also moves the step sequence) is accurate to ~1e-6.  The start times and
    the RSA/UFA switch times are numerical choices that forward-mode AD does not
    differentiate (a bisection root and lax.cond branches in the reference); the shifted
    solves hold them at the base point's values, so the quotient measures the same
    derivative (letting them move changes it by ~1e-3: the adiabatic initial conditions and
    the approximations are accurate to that level, not to round-off).  The shifted backgrounds replay the Recfast step sequence of the base point: Recfast runs its
    own adaptive solve at rtol 1e-3, whose step choices would put ~1e-7 relative noise in x_e
    (~1e-3 in a difference quotient of step 1e-4); forward-mode AD, as the reference applies
    it, differentiates the discrete background with those choices held, and so does the
    replay.  The Recfast switches (jnp.where on x_H, x_He in the reference) make the
    background piecewise smooth; the jumps they leave in P are ~1e-8 relative.
    """
    from discoeb_b200.gradients import THETA_NAMES, power_spectrum_jacobian
    solver = dict(rtol=1e-10, atol=1e-13, max_steps=400000)
    k, P, J = power_spectrum_jacobian(THETA, aexp_out=(0.5, 1.0), kmin=1e-3, kmax=0.5, num_k=8, **solver, **L143)
    assert P.shape == (8, 2) and J.shape == (8, 8, 2)
    from discoeb_b200.perturbations import approximation_switch_times, determine_starting_time
    trace = {}
    P0, bg = _power(THETA, k, (0.5, 1.0), trace=trace, **solver)
    np.testing.assert_allclose(P, P0, rtol=1e-8)  # same algorithm, solver tolerance 1e-10
    tau_out = bg["tau_of_a_spline"].evaluate(np.array([0.5, 1.0]))
    fixed = dict(tau_start=0.99 * np.minimum(tau_out.min(), determine_starting_time(param=bg, k=k)),
                 switch_tau=approximation_switch_times(bg, k))
    worst = {}
    for i, name in enumerate(THETA_NAMES):
        eps = 1e-4 * abs(THETA[name])
        tp, tm = dict(THETA), dict(THETA)
        tp[name] += eps
        tm[name] -= eps
        fd = (_power(tp, k, (0.5, 1.0), replay=trace, **fixed, **solver)[0]
              - _power(tm, k, (0.5, 1.0), replay=trace, **fixed, **solver)[0]) / (2 * eps)
        err = np.abs(J[i] - fd) / (np.abs(fd) + 1e-3 * np.abs(fd).max())
        worst[name] = float(err.max())
    assert max(worst.values()) < 2e-4, worst


def test_gpu_autograd_function_contracts_the_jacobian(torch_cuda):
    torch = torch_cuda
    from discoeb_b200.gradients import THETA_NAMES, power_spectrum_function, power_spectrum_jacobian
    opts = dict(aexp_out=(1.0,), kmin=1e-3, kmax=0.3, num_k=6, **L143)
    PK = power_spectrum_function(**opts)
    theta = torch.tensor([THETA[n] for n in THETA_NAMES], dtype=torch.float64, device="cuda", requires_grad=True)
    P = PK.apply(theta)
    weights = torch.linspace(0.5, 2.0, P.numel(), dtype=torch.float64, device="cuda").reshape(P.shape)
    (P * weights).sum().backward()
    _, P_ref, J = power_spectrum_jacobian(THETA, **opts)
    np.testing.assert_allclose(P.detach().cpu().numpy(), P_ref, rtol=1e-12)
    expect = np.einsum("dkn,kn->d", J, weights.cpu().numpy())
    np.testing.assert_allclose(theta.grad.cpu().numpy(), expect, rtol=1e-12)


def test_gpu_jvp_records_in_global_memory_equal_the_shared_form(torch_cuda):
    """l_max 50 (n = 219): the shared-memory step records leave room for three tangent warps per
    block, so discoeb_jvp_records keeps them in a global workspace and runs all six directions in
    one block; same code on the same steps, so the same states and tangents as the plain entry
    (which splits the directions over two blocks, each with its own forward)"""
    import ctypes
    from discoeb_b200.gradients import JacobianProblem
    L50 = dict(lmaxg=50, lmaxgp=50, lmaxr=17, lmaxnu=17, nqmax=5)
    prob = JacobianProblem(THETA, aexp_out=np.array([0.2, 0.5, 1.0]), kmodes=np.geomspace(1e-3, 0.3, 5), rtol=1e-5,
                           atol=1e-8, full_state=True, **L50)
    assert prob.lib.discoeb_jvp_records_bytes(ctypes.byref(prob.dc.host), 6, prob.K) > 0
    prob.launch(records=False)
    y, yd = prob.d_out.clone(), prob.d_outd.clone()
    prob.launch()
    np.testing.assert_array_equal(prob.d_out.cpu().numpy(), y.cpu().numpy())
    np.testing.assert_array_equal(prob.d_outd.cpu().numpy(), yd.cpu().numpy())
    assert np.isfinite(yd.cpu().numpy()).all()
    # n = 143 gains nothing: every direction already shares the block
    p143 = JacobianProblem(THETA, aexp_out=A4, kmodes=np.geomspace(1e-3, 0.3, 5), rtol=1e-5, atol=1e-8, **L143)
    assert p143.lib.discoeb_jvp_records_bytes(ctypes.byref(p143.dc.host), 6, p143.K) == 0
