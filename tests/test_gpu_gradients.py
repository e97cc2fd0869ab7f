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


def _power(theta, kmodes, aexp_out, **solver):
    """P(k) of the forward path (evolve_background + solve_modes + get_power)."""
    from discoeb_b200.background import evolve_background
    from discoeb_b200.gradients import theta_to_params
    from discoeb_b200.perturbations import get_power, solve_modes
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        bg = evolve_background(param=theta_to_params(theta))
    tout = bg["tau_of_a_spline"].evaluate(np.asarray(aexp_out, dtype=np.float64))
    y = solve_modes(param=bg, kmodes=kmodes, tau_out=tout, pcoeff=0.25, icoeff=0.8, dcoeff=0.0, factormax=20.0,
                    factormin=0.3, return_full=False, **solver, **L143)
    return get_power(k=kmodes[:, None], y=y, idx=4, param=bg)


def test_gpu_jvp_values_match_forward_solve(torch_cuda):
    from discoeb_b200.gradients import JacobianProblem
    prob = JacobianProblem(THETA, aexp_out=A4, kmin=1e-4, kmax=10.0, num_k=24, rtol=1e-5, atol=1e-8, **L143)
    prob.launch()
    P, J, status, nsteps = prob.result()
    assert (status == 0).all()
    P_fwd = _power(THETA, prob.kmodes, A4, rtol=1e-5, atol=1e-8, max_steps=100000)
    # same algorithm and step sequence: the value part of the tangent solve is the forward solve
    np.testing.assert_allclose(P, P_fwd, rtol=1e-9)
    assert np.isfinite(J).all()


def test_gpu_jacobian_matches_central_differences(torch_cuda):
    """dP/dtheta against central differences with relative step 1e-4.

    Both sides run at rtol 1e-10 so that the difference quotient of the adaptive solve
    (which also moves the start times and the step sequence) is accurate to ~1e-6.  The
    Recfast switches (jnp.where on x_H, x_He in the reference) make the background a
    piecewise-smooth function of theta; the jumps they leave in P are ~1e-8 relative.
    """
    from discoeb_b200.gradients import THETA_NAMES, power_spectrum_jacobian
    solver = dict(rtol=1e-10, atol=1e-13, max_steps=400000)
    k, P, J = power_spectrum_jacobian(THETA, aexp_out=(0.5, 1.0), kmin=1e-3, kmax=0.5, num_k=8, **solver, **L143)
    assert P.shape == (8, 2) and J.shape == (8, 8, 2)
    worst = {}
    for i, name in enumerate(THETA_NAMES):
        eps = 1e-4 * abs(THETA[name])
        tp, tm = dict(THETA), dict(THETA)
        tp[name] += eps
        tm[name] -= eps
        fd = (_power(tp, k, (0.5, 1.0), **solver) - _power(tm, k, (0.5, 1.0), **solver)) / (2 * eps)
        err = np.abs(J[i] - fd) / (np.abs(fd) + 1e-3 * np.abs(fd).max())
        worst[name] = float(err.max())
    assert max(worst.values()) < 2e-4, worst
