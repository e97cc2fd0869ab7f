"""discoeb_background_batch (the background, Recfast and their tangents of many cosmologies in one
GPU launch) against the host entry discoeb_background (GPU)."""
import warnings

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("no CUDA device: the -m gpu tests need a GPU")
    return torch


def _scaled_err(a, b, floor=0.0):
    """max |a - b| over the finite entries (which must coincide) / max(max |b|, floor)"""
    a, b = np.asarray(a), np.asarray(b)
    f = np.isfinite(b)
    assert np.array_equal(f, np.isfinite(a))
    if not f.any():
        return 0.0
    return float(np.abs(a[f] - b[f]).max() / max(np.abs(b[f]).max(), floor, 1e-300))


def test_gpu_background_batch_matches_host(torch_cuda):
    from discoeb_b200 import _abi
    from discoeb_b200.background import native_background, native_backgrounds_device
    from discoeb_b200.gradients import ODE_DIRECTIONS, param_dots, theta_to_params
    from discoeb_b200.workloads import sample_thetas, workload
    thetas = [workload("pk_lcdm_mnu_k512_z4")["theta"]] + sample_thetas(3, seed=11)
    params = [theta_to_params(t) for t in thetas]
    dots = [param_dots(t, ODE_DIRECTIONS) for t in thetas]
    out, out_dot = native_backgrounds_device(params, 256, dots)
    out, out_dot = out.cpu().numpy(), out_dot.cpu().numpy()
    v_only = native_backgrounds_device(params, 256)[0].cpu().numpy()
    lay, _ = _abi.background_layout(256)
    # Recfast-independent fields (densities, neutrino tables, conformal times) agree to the last bits
    # of the device's exp/log/pow; downstream of Recfast the reference's cancelling Saha x_H formula
    # amplifies such bits (to ~1e-6 of the values' scale), and its rounding-noise slope xeprime_recf
    # is left out, as between the host restatements
    smooth = {"t:aexp", "t:loga", "t:tau", "t:tau_of_a_S", "t:a_of_tau_S"}
    for c, (p, d) in enumerate(zip(params, dots)):
        buf, bdot = native_background(p, 256, d)
        # the same Recfast branches and step counts in every interval, in the value pass and in the
        # tangent passes (whose value parts differ from the value pass only where the device
        # compiler contracts the two instantiations' multiply-adds differently)
        for o in (out[c], v_only[c]):
            np.testing.assert_array_equal(o[lay["t:rec_case"]], buf[lay["t:rec_case"]])
            np.testing.assert_array_equal(o[lay["t:rec_steps"]], buf[lay["t:rec_steps"]])
        bad = {}
        for key, sl in lay.items():
            if key in ("t:xeprime_recf", "t:rec_case", "t:rec_steps"):
                continue
            tight = key.startswith("n:") or key in smooth or (key.startswith("s:") and key != "s:tau_maxvis")
            vtol, ttol = (1e-10, 1e-8) if tight else (1e-5, 1e-4)
            verr = max(_scaled_err(out[c][sl], buf[sl]), _scaled_err(v_only[c][sl], buf[sl]))
            # a tangent that vanishes analytically (d opac / d h: opac depends on omega_b = Omegab h^2
            # only) is rounding noise on both sides: its scale has a floor of 1e-8 of the values'
            vscale = np.abs(buf[sl][np.isfinite(buf[sl])]).max(initial=0.0)
            terr = max(_scaled_err(out_dot[c, j][sl], bdot[j][sl], 1e-8 * vscale) for j in range(len(dots[c])))
            if verr >= vtol or terr >= ttol:
                bad[key] = (verr, terr)
        assert not bad, (c, bad)


def test_gpu_background_batch_in_the_batched_prologues(torch_cuda):
    from discoeb_b200.background import evolve_background
    from discoeb_b200.gradients import JacobianBatch, theta_to_params
    from discoeb_b200.perturbations import backgrounds
    from discoeb_b200.workloads import crosses_phantom_divide, sample_thetas
    # cosmologies whose w(a) stays on one side of -1: at a crossing the dark-energy equations are
    # singular and the solve amplifies any input difference, last bits included
    thetas = [t for t in sample_thetas(12, seed=5) if not crosses_phantom_divide(t)][:3]
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        host = [evolve_background(param=theta_to_params(t)) for t in thetas]
    dev = backgrounds([theta_to_params(t) for t in thetas], device="cuda")
    for a, b in zip(dev, host):
        assert set(a) == set(b)
        np.testing.assert_allclose(a["tau"], b["tau"], rtol=1e-12)
        np.testing.assert_allclose(a["xe"], b["xe"], rtol=1e-5)
    ks = np.geomspace(1e-3, 0.5, 12)
    kw = dict(kmodes=ks, aexp_out=np.array([1.0]), lmaxg=12, lmaxgp=12, lmaxr=17, lmaxnu=17, nqmax=5)
    P, J = [], []
    for hb in ("native", "device"):
        jb = JacobianBatch(thetas, host_backend=hb, **kw)
        jb.launch()
        p, j, st, _ = jb.result()
        assert (st == 0).all()
        P.append(p)
        J.append(j)
    # the backgrounds differ in their last bits (x_e by up to ~1e-6 where Recfast's Saha formula
    # cancels), which the solve carries to P(k) and its Jacobian at about the solver tolerance
    np.testing.assert_allclose(P[1], P[0], rtol=1e-5)
    assert np.abs(J[1] - J[0]).max() <= 1e-4 * np.abs(J[0]).max()
