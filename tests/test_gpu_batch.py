"""Several cosmologies in one discoeb_fwd launch (perturbations.solve_cosmologies) against one
launch per cosmology, and the kernel's own check of the cosmology index."""
import ctypes
import warnings

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

L65 = dict(lmaxg=12, lmaxgp=12, lmaxr=17, lmaxnu=3, nqmax=3)


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("no CUDA device: the -m gpu tests need a GPU")
    return torch


def test_gpu_batch_equals_single_cosmology_launches(torch_cuda):
    from discoeb_b200.background import evolve_background
    from discoeb_b200.gradients import theta_to_params
    from discoeb_b200.perturbations import solve_cosmologies, solve_modes
    from discoeb_b200.workloads import sample_thetas
    thetas = [t for t in sample_thetas(12, seed=3)][:3]
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        bgs = [evolve_background(param=theta_to_params(t)) for t in thetas]
    ks = np.geomspace(1e-3, 1.0, 6)
    aout = np.array([0.5, 1.0])
    kw = dict(rtol=1e-5, atol=1e-8, max_steps=100000, **L65)
    yb, st, ns = solve_cosmologies(params=bgs, kmodes=ks, aexp_out=aout, return_stats=True, on_failure="ignore", **kw)
    assert yb.shape == (3, 6, 2, 20)
    for c, bg in enumerate(bgs):
        tout = bg["tau_of_a_spline"].evaluate(aout)
        y1, s1, n1 = solve_modes(param=bg, kmodes=ks, tau_out=tout, pcoeff=0.25, icoeff=0.8, dcoeff=0.0,
                                 factormax=20.0, factormin=0.3, return_full=False, return_stats=True,
                                 on_failure="ignore", **kw)
        np.testing.assert_array_equal(st[c], s1)
        np.testing.assert_array_equal(ns[c], n1)
        np.testing.assert_array_equal(yb[c], y1)  # same per-mode computation, bit for bit


def test_gpu_bad_cosmology_index_is_reported(torch_cuda):
    torch = torch_cuda
    from conftest import background
    from discoeb_b200 import _abi
    from discoeb_b200.perturbations import (DeviceCosmo, adiabatic_ics, approximation_switch_times,
                                            determine_starting_time)
    bg = background("lcdm_massless", 256)
    dc = DeviceCosmo(bg, de_guard_eps=1e-9, device=torch.device("cuda"), **L65)
    ks = np.array([0.1, 0.01])
    tout = bg["tau_of_a_spline"].evaluate(np.array([1.0]))
    t0 = 0.99 * np.minimum(tout.min(), determine_starting_time(param=bg, k=ks))
    f = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    y0 = f(adiabatic_ics(tau=t0, param=bg, kmode=ks, **L65))
    out = torch.zeros((2, 1, 20), dtype=torch.float64, device="cuda")
    stat = torch.zeros((2, 2), dtype=torch.int32, device="cuda")
    mc = f(np.array([0, 7], dtype=np.int32))  # the second mode names a cosmology that does not exist
    ctrl = _abi.DiscoebControl(1e-5, 1e-8, 0.25, 0.8, 0.0, 20.0, 0.3, 100000, 0, 0, 0)
    # keep every device input referenced until the kernel has finished
    d_k, d_t0, d_sw, d_tout = f(ks), f(t0), f(approximation_switch_times(bg, ks)), f(tout)
    rc = _abi.lib().discoeb_fwd(dc.struct.data_ptr(), ctypes.byref(dc.host), 1, ctypes.byref(ctrl), 2, mc.data_ptr(),
                                d_k.data_ptr(), d_t0.data_ptr(), y0.data_ptr(), d_sw.data_ptr(), 1,
                                d_tout.data_ptr(), None, out.data_ptr(), stat[0].data_ptr(), stat[1].data_ptr(),
                                torch.cuda.current_stream().cuda_stream)
    assert rc == 0
    s = stat.cpu().numpy()
    assert s[0, 0] == 0 and s[0, 1] == 5 and s[1, 1] == 0
    o = out.cpu().numpy()
    assert np.isfinite(o[0]).all() and np.isnan(o[1]).all()


def test_gpu_jacobian_batch_equals_single_cosmology_launches(torch_cuda):
    from discoeb_b200.gradients import JacobianBatch, JacobianProblem
    from discoeb_b200.workloads import sample_thetas
    thetas = sample_thetas(2, seed=11)
    ks = np.geomspace(1e-3, 0.5, 5)
    kw = dict(aexp_out=(0.5, 1.0), rtol=1e-5, atol=1e-8, **L65)
    batch = JacobianBatch(thetas, kmodes=ks, host_processes=1, **kw)
    batch.launch()
    P, J, status, nsteps = batch.result(on_failure="ignore")
    assert P.shape == (2, 5, 2) and J.shape == (2, 8, 5, 2)
    for c, th in enumerate(thetas):
        one = JacobianProblem(th, kmodes=ks, **kw)
        one.launch()
        P1, J1, s1, n1 = one.result(on_failure="ignore")
        np.testing.assert_array_equal(status[c], s1)
        np.testing.assert_array_equal(nsteps[c], n1)
        np.testing.assert_array_equal(P[c], P1)  # same per-mode arithmetic in both launches
        np.testing.assert_array_equal(J[c], J1)
