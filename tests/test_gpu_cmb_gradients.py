"""dC_l/dtheta (cmb.compute_Cell_jacobian: discoeb_jvp_full plus directional differences of the
deterministic stages after the solve) against the forward chain and against central finite
differences of the whole chain (GPU)."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

THETA = dict(omega_c=0.120, omega_b=0.0224, h=0.674, n_s=0.965, ln10As=math.log(21.0), w0=-0.95, wa=0.05, m_nu=0.06)
# a reduced chain: 32 camb-sampled modes, l <= 600, 1024 dense modes, 4096 FFTLog points; and the
# reference's pipeline defaults
SMALL = dict(ellmax=600, nmodes=32, n_k_dense=1024, n_fftlog=4096)
DEFAULT = dict(ellmax=2500, nmodes=128, n_k_dense=8192, n_fftlog=16384)
NO_DENSE = dict(ellmax=600, nmodes=32, n_k_dense=0, n_fftlog=4096)  # the modes' own k grid


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("no CUDA device: the -m gpu tests need a GPU")
    return torch


def _chain(bg, kmodes, solver, fixed, size):
    """C_l of the forward chain (full solve, sources, line of sight, C_l) on the background dict
    ``bg`` at fixed k sampling, start times and switch times."""
    from discoeb_b200 import cmb
    from discoeb_b200.perturbations import solve_modes
    a = cmb.cmb_aexp_out()
    tau = bg["tau_of_a_spline"].evaluate(a)
    L = dict(lmaxg=11, lmaxgp=11, lmaxr=11, lmaxnu=8, nqmax=3)
    y = solve_modes(param=bg, kmodes=kmodes, tau_out=tau, pcoeff=0.25, icoeff=0.8, dcoeff=0.0, factormax=20.0,
                    factormin=0.3, return_full=True, as_tensor=True, **fixed, **solver, **L)
    src = cmb.compute_sources(param=bg, yout=y, kmodes=kmodes, aexp_out=a, **L)
    th, kk = cmb.compute_theta_ell(size["ellmax"], kmodes, tau, src["S"], float(bg["tau_of_a_spline"].evaluate(1.0)),
                                   n_fftlog=size["n_fftlog"], n_k_dense=size["n_k_dense"])
    return cmb.compute_Cell(th, kk, bg["n_s"], bg["k_p"]).cpu().numpy()


@pytest.mark.parametrize("size", [SMALL, DEFAULT], ids=["small", "reference_defaults"])
def test_gpu_cell_jacobian_matches_central_differences(torch_cuda, size):
    """dC_l/dtheta against fourth-order central differences (step 1e-4 of each parameter) of the
    forward chain at solver rtol 1e-11, on backgrounds moved along the exact background tangent.

    Fourth order because the discrete C_l has a fast ripple in the parameters: the FFTLog grid in
    ln(tau0 - tau) moves with tau0, and the line of sight's discretisation error is periodic in
    the grid's offset (one cell, 2.4e-3 in ln chi at 4096 points, is a ~2e-3 relative change of
    omega_c); the exact derivative of the discrete chain contains the ripple's slope, which a
    second-order quotient of step 1e-4 misses by ~4e-4.

    The background enters as its forward-mode tangent (discoeb_background, checked against the
    complex-step derivative of the numpy restatement in the CPU tests): a difference quotient of
    Recfast itself carries the rounding of the reference's cancelling Saha x_H formula (x_e moves
    by up to ~1e-6 of its scale between two evaluations an ulp apart, ~1e-2 in a quotient of
    step 1e-4 in the He recombination era), which C_l, unlike P(k), feels.  The start and switch
    times are held, as forward-mode AD through the reference holds them; everything else, the
    solve included, is differenced."""
    from discoeb_b200.background import _DIFF_FIELDS, background_from_buffer, native_background
    from discoeb_b200.cmb import compute_Cell_jacobian
    from discoeb_b200.gradients import ODE_DIRECTIONS, THETA_NAMES, param_dots, theta_to_params
    from discoeb_b200.perturbations import approximation_switch_times, determine_starting_time, k_sampling
    from discoeb_b200 import cmb
    # rtol 1e-11: the quotient re-runs the adaptive solve, whose step sequence can change between
    # the four points; at 1e-9 that noise, over a step of 1e-4, reached ~2e-4 of the weakest
    # directions' derivative on some backgrounds
    solver = dict(rtol=1e-11, atol=1e-14, max_steps=2000000)
    C, J, param = compute_Cell_jacobian(THETA, **size, **solver)
    assert C.shape == (size["ellmax"] + 1,) and J.shape == (8, size["ellmax"] + 1)
    assert np.isfinite(J).all()
    assert np.all(J[THETA_NAMES.index("ln10As")] == 0.0)
    p = theta_to_params(THETA)
    pd = param_dots(THETA, ODE_DIRECTIONS)
    buf, bd = native_background(p, 1024, pd)
    bg = background_from_buffer(p, buf, 1024)
    kmodes = k_sampling(bg, 1e-4, 1.0, size["nmodes"], "camb")
    tau_out = bg["tau_of_a_spline"].evaluate(cmb.cmb_aexp_out())
    fixed = dict(tau_start=0.99 * np.minimum(tau_out.min(), determine_starting_time(param=bg, k=kmodes)),
                 switch_tau=approximation_switch_times(bg, kmodes))
    l = slice(2, None)
    # the same chain at the same background: the jvp and forward kernels differ in compiled rounding
    np.testing.assert_allclose(C[l], _chain(bg, kmodes, solver, fixed, size)[l], rtol=1e-7)
    worst = {}
    for i, name in enumerate(THETA_NAMES):
        if name == "ln10As":
            continue
        eps = 1e-4 * abs(THETA[name])
        fd = 0.0
        for sgn, wgt in ((2.0, -1.0 / 12.0), (1.0, 8.0 / 12.0), (-1.0, -8.0 / 12.0), (-2.0, 1.0 / 12.0)):
            if name == "n_s":
                b = dict(bg)
                b["n_s"] = bg["n_s"] + sgn * eps
            else:
                di = ODE_DIRECTIONS.index(name)
                ps = dict(p)
                for f in _DIFF_FIELDS:
                    ps[f] = p[f] + sgn * eps * pd[di][f]
                b = background_from_buffer(ps, buf + sgn * eps * bd[di], 1024)
            fd = fd + wgt * _chain(b, kmodes, solver, fixed, size) / eps
        # dC_l/dtheta oscillates in l and crosses zero: deviations against the direction's largest
        worst[name] = float(np.abs(J[i][l] - fd[l]).max() / np.abs(fd[l]).max())
    print("max |J - fd| / max |fd| per direction:", worst)
    # measured: <= 4e-6 on the reduced chain; at the reference's defaults <= 2.6e-5 except m_nu
    # (7.1e-5), limited by the check itself: its step-1e-4 quotient misses ~2e-5 of the ripple
    # (a cell of the 16384-point grid is ~1.2e-3 of omega_c), and in the directions C_l is least
    # sensitive to the solver's rounding in the quotient weighs most.  Bound: the metric's 1e-4
    assert max(worst.values()) < 1e-4, worst


def test_gpu_cell_jacobian_does_not_depend_on_the_difference_step(torch_cuda):
    """The stages after the solve are smooth along the exact tangent: their fourth-order
    differences with steps 1e-4 and 3e-4 (relative) agree far below the solver tolerance (a
    source point whose approximation regime, evaluated from its own time and scale factor as in
    the reference's compute_time_derivatives, changes inside the wider stencil leaves ~1e-6)."""
    from discoeb_b200.cmb import compute_Cell_jacobian
    C1, J1, _ = compute_Cell_jacobian(THETA, rel_step=1e-4, **SMALL)
    C2, J2, _ = compute_Cell_jacobian(THETA, rel_step=3e-4, **SMALL)
    np.testing.assert_array_equal(C1, C2)
    l = slice(2, None)
    dev = [float(np.abs(J1[i][l] - J2[i][l]).max() / max(np.abs(J1[i][l]).max(), 1e-300)) for i in range(8)]
    print("step dependence per direction:", dev)
    assert max(dev) <= 1e-5, dev


@pytest.mark.parametrize("size", [SMALL, DEFAULT, NO_DENSE], ids=["small", "reference_defaults", "no_dense_k"])
def test_gpu_line_of_sight_tangent_equals_its_differences(torch_cuda, size):
    """The forward-mode line of sight (discoeb_los_cell_jvp) against fourth-order differences of
    the same line of sight along the same first-order path: one derivative, two evaluations.

    The differences' truncation error is (omega h)^4 / 30 of the ripple's share of the derivative,
    omega the ripple's frequency in the parameter (one FFTLog cell per period: at 16384 points a
    period is ~1.2e-3 of omega_c, so step 1e-4 leaves ~2e-5); at step 2.5e-5 it is 256 times
    smaller, but the rounding of the line of sight (its FFTLog sum cancels at low l) over the
    step grows 4 times and takes over in the directions C_l is least sensitive to.  Per direction
    the better of the two steps is compared (measured: <= 8e-6 at the reference's defaults,
    <= 1.3e-6 on the reduced chain)."""
    from discoeb_b200.cmb import compute_Cell_jacobian
    C1, J1, _ = compute_Cell_jacobian(THETA, los="tangent", **size)
    l = slice(2, None)
    devs = []
    for step in (1e-4, 2.5e-5):
        C2, J2, _ = compute_Cell_jacobian(THETA, los="differences", rel_step=step, **size)
        np.testing.assert_array_equal(C1, C2)
        devs.append([float(np.abs(J1[i][l] - J2[i][l]).max() / max(np.abs(J2[i][l]).max(), 1e-300)) for i in range(8)])
    print("tangent vs differences (steps 1e-4, 2.5e-5) per direction:", devs)
    best = [min(a, b) for a, b in zip(*devs)]
    assert max(best) <= 2e-5, best


def test_gpu_cell_autograd_function_contracts_the_jacobian(torch_cuda):
    torch = torch_cuda
    from discoeb_b200.cmb import cell_spectrum_function, compute_Cell_jacobian
    from discoeb_b200.gradients import THETA_NAMES
    CS = cell_spectrum_function(**SMALL)
    theta = torch.tensor([THETA[n] for n in THETA_NAMES], dtype=torch.float64, device="cuda", requires_grad=True)
    C = CS.apply(theta)
    weights = torch.linspace(0.5, 2.0, C.numel(), dtype=torch.float64, device="cuda")
    (C * weights).sum().backward()
    C_ref, J, _ = compute_Cell_jacobian(THETA, **SMALL)
    np.testing.assert_array_equal(C.detach().cpu().numpy(), C_ref)
    np.testing.assert_allclose(theta.grad.cpu().numpy(), J @ weights.cpu().numpy(), rtol=1e-12)


@pytest.mark.parametrize("size", [SMALL, DEFAULT], ids=["small", "reference_defaults"])
def test_gpu_forward_mode_sources_equal_their_differences(torch_cuda, size):
    """discoeb_sources_jvp (the sources' derivative in dual numbers) against the central difference
    of the whole source stage along the same tangents (O(h^2) with h = 1e-4 of each parameter)."""
    from discoeb_b200.cmb import compute_Cell_jacobian
    C1, J1, _ = compute_Cell_jacobian(THETA, sources="tangent", **size)
    C2, J2, _ = compute_Cell_jacobian(THETA, sources="differences", **size)
    np.testing.assert_array_equal(C1, C2)
    l = slice(2, None)
    dev = [float(np.abs(J1[i][l] - J2[i][l]).max() / max(np.abs(J2[i][l]).max(), 1e-300)) for i in range(8)]
    print("forward-mode vs differenced sources per direction:", dev)
    assert max(dev) <= 1e-6, dev


def _chain_pol(bg, kmodes, solver, fixed, size):
    """C_l^TE and C_l^EE of the forward chain on the background dict ``bg`` (as _chain)."""
    from discoeb_b200 import cmb
    from discoeb_b200.perturbations import solve_modes
    a = cmb.cmb_aexp_out()
    tau = bg["tau_of_a_spline"].evaluate(a)
    tau0 = float(bg["tau_of_a_spline"].evaluate(1.0))
    L = dict(lmaxg=11, lmaxgp=11, lmaxr=11, lmaxnu=8, nqmax=3)
    y = solve_modes(param=bg, kmodes=kmodes, tau_out=tau, pcoeff=0.25, icoeff=0.8, dcoeff=0.0, factormax=20.0,
                    factormin=0.3, return_full=True, as_tensor=True, **fixed, **solver, **L)
    src = cmb.compute_sources(param=bg, yout=y, kmodes=kmodes, aexp_out=a, **L)
    kw = dict(n_fftlog=size["n_fftlog"], n_k_dense=size["n_k_dense"])
    tht, kk = cmb.compute_theta_ell(size["ellmax"], kmodes, tau, src["S"], tau0, **kw)
    the, _ = cmb.compute_theta_ell(size["ellmax"], kmodes, tau, src["E"], tau0, kind="E", **kw)
    return {"TE": cmb.compute_Cell(tht, kk, bg["n_s"], bg["k_p"], theta_ell_b=the).cpu().numpy(),
            "EE": cmb.compute_Cell(the, kk, bg["n_s"], bg["k_p"]).cpu().numpy()}


def test_gpu_polarisation_jacobian_matches_central_differences(torch_cuda):
    """dC_l^TE/dtheta and dC_l^EE/dtheta (the E source's tangent from discoeb_sources_jvp, the
    E-mode line of sight by fourth-order differences along the path) against fourth-order central
    differences of the whole chain at solver rtol 1e-11 on the reduced chain, as the TT test does;
    and the TT block of the same call equals the TT-only call."""
    from discoeb_b200.background import _DIFF_FIELDS, background_from_buffer, native_background
    from discoeb_b200.cmb import compute_Cell_jacobian
    from discoeb_b200.gradients import ODE_DIRECTIONS, THETA_NAMES, param_dots, theta_to_params
    from discoeb_b200.perturbations import approximation_switch_times, determine_starting_time, k_sampling
    from discoeb_b200 import cmb
    solver = dict(rtol=1e-11, atol=1e-14, max_steps=2000000)
    size = SMALL
    C, J, _ = compute_Cell_jacobian(THETA, spectra=("TT", "TE", "EE"), **size, **solver)
    assert set(C) == {"TT", "TE", "EE"}
    C_tt, J_tt, _ = compute_Cell_jacobian(THETA, **size, **solver)
    np.testing.assert_array_equal(C["TT"], C_tt)
    np.testing.assert_array_equal(J["TT"], J_tt)
    p = theta_to_params(THETA)
    pd = param_dots(THETA, ODE_DIRECTIONS)
    buf, bd = native_background(p, 1024, pd)
    bg = background_from_buffer(p, buf, 1024)
    kmodes = k_sampling(bg, 1e-4, 1.0, size["nmodes"], "camb")
    tau_out = bg["tau_of_a_spline"].evaluate(cmb.cmb_aexp_out())
    fixed = dict(tau_start=0.99 * np.minimum(tau_out.min(), determine_starting_time(param=bg, k=kmodes)),
                 switch_tau=approximation_switch_times(bg, kmodes))
    base = _chain_pol(bg, kmodes, solver, fixed, size)
    l = slice(2, None)
    for sp in ("TE", "EE"):
        np.testing.assert_allclose(C[sp][l], base[sp][l], rtol=1e-7, atol=1e-7 * np.abs(base[sp][l]).max())
        assert np.isfinite(J[sp]).all() and np.all(J[sp][THETA_NAMES.index("ln10As")] == 0.0)
    worst = {"TE": {}, "EE": {}}
    for i, name in enumerate(THETA_NAMES):
        if name == "ln10As":
            continue
        eps = 1e-4 * abs(THETA[name])
        fd = {"TE": 0.0, "EE": 0.0}
        for sgn, wgt in ((2.0, -1.0 / 12.0), (1.0, 8.0 / 12.0), (-1.0, -8.0 / 12.0), (-2.0, 1.0 / 12.0)):
            if name == "n_s":
                b = dict(bg)
                b["n_s"] = bg["n_s"] + sgn * eps
            else:
                di = ODE_DIRECTIONS.index(name)
                ps = dict(p)
                for f in _DIFF_FIELDS:
                    ps[f] = p[f] + sgn * eps * pd[di][f]
                b = background_from_buffer(ps, buf + sgn * eps * bd[di], 1024)
            ch = _chain_pol(b, kmodes, solver, fixed, size)
            for sp in fd:
                fd[sp] = fd[sp] + wgt * ch[sp] / eps
        for sp in fd:
            # TE crosses zero in l: deviations against the direction's largest
            worst[sp][name] = float(np.abs(J[sp][i][l] - fd[sp][l]).max() / np.abs(fd[sp][l]).max())
    print("max |J - fd| / max |fd| per direction:", worst)
    assert max(max(w.values()) for w in worst.values()) < 1e-4, worst


def test_gpu_polarisation_forward_mode_sources_equal_their_differences(torch_cuda):
    """The E source's forward-mode tangent (discoeb_sources_jvp's SE_dot) against the central
    difference of the whole source stage along the same tangents, through C_l^TE and C_l^EE."""
    from discoeb_b200.cmb import compute_Cell_jacobian
    C1, J1, _ = compute_Cell_jacobian(THETA, sources="tangent", spectra=("TE", "EE"), **SMALL)
    C2, J2, _ = compute_Cell_jacobian(THETA, sources="differences", spectra=("TE", "EE"), **SMALL)
    l = slice(2, None)
    for sp in ("TE", "EE"):
        np.testing.assert_array_equal(C1[sp], C2[sp])
        dev = [float(np.abs(J1[sp][i][l] - J2[sp][i][l]).max() / max(np.abs(J2[sp][i][l]).max(), 1e-300))
               for i in range(8)]
        print(sp, "forward-mode vs differenced sources per direction:", dev)
        assert max(dev) <= 1e-6, (sp, dev)


def test_gpu_sources_jvp_batched_directions_equal_single_calls(torch_cuda):
    """discoeb_sources_jvp with all six directions in one call (one warp per mode and time, the
    base point's y' once) gives the same source tangents, bit for bit, as one call per direction"""
    import ctypes

    import torch
    from discoeb_b200 import _abi
    from discoeb_b200.cmb import background_table, cmb_aexp_out, compute_sources
    from discoeb_b200.gradients import JacobianProblem
    L = dict(lmaxg=11, lmaxgp=11, lmaxr=11, lmaxnu=8, nqmax=3)
    theta = dict(omega_c=0.120, omega_b=0.0224, h=0.674, n_s=0.965, ln10As=math.log(21.0), w0=-0.95, wa=0.05,
                 m_nu=0.06)
    a = cmb_aexp_out()
    ks = np.geomspace(1e-3, 0.2, 6)
    prob = JacobianProblem(theta, aexp_out=a, kmodes=ks, rtol=1e-4, atol=1e-4, full_state=True, num_thermo=1024, **L)
    prob.launch()
    y, k_rows, _ = prob.launch_states()
    bg = prob.bg
    tau = bg["tau_of_a_spline"].evaluate(a)
    dev = y.device
    f = compute_sources(param=bg, yout=y, kmodes=k_rows, aexp_out=a, device=dev, **L)
    K, T = f["S"].shape
    rng = np.random.default_rng(5)
    tau_dot = torch.from_numpy(rng.standard_normal((6, T)) * 1e-2).to(dev)
    bt = torch.from_numpy(background_table(a, tau, bg)).to(dev)
    bt_dot = torch.from_numpy(rng.standard_normal((6,) + tuple(bt.shape)) * 1e-3 * np.abs(bt.cpu().numpy())).to(dev)
    d_k = torch.from_numpy(np.ascontiguousarray(k_rows)).to(dev)
    d_tau = torch.from_numpy(np.ascontiguousarray(tau)).to(dev)
    lib = _abi.lib()
    tan_size = ctypes.sizeof(_abi.DiscoebTangent)
    stream = torch.cuda.current_stream(dev).cuda_stream

    def call(d0, nd):
        S = torch.empty((nd, K, T), dtype=torch.float64, device=dev)
        SE = torch.empty((nd, K, T), dtype=torch.float64, device=dev)
        scratch = torch.empty(8 * nd * K * T, dtype=torch.float64, device=dev)
        rc = lib.discoeb_sources_jvp(prob.dc.struct.data_ptr(), ctypes.byref(prob.dc.host),
                                     prob.d_tan.data_ptr() + d0 * tan_size, nd, K, d_k.data_ptr(), T, d_tau.data_ptr(),
                                     tau_dot[d0:d0 + nd].contiguous().data_ptr(), bt.data_ptr(),
                                     bt_dot[d0:d0 + nd].contiguous().data_ptr(), y.data_ptr(),
                                     prob.d_outd[d0:d0 + nd].contiguous().data_ptr(), f["S"].data_ptr(), S.data_ptr(),
                                     scratch.data_ptr(), SE.data_ptr(), stream)
        assert rc == 0
        return S.cpu().numpy(), SE.cpu().numpy()

    S6, SE6 = call(0, 6)
    for d in range(6):
        S1, SE1 = call(d, 1)
        np.testing.assert_array_equal(S6[d], S1[0])
        np.testing.assert_array_equal(SE6[d], SE1[0])
    assert np.isfinite(S6).all() and np.abs(S6).max() > 0
