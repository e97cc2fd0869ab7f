"""discoeb_background (C++ background + Recfast with forward-mode tangents) against the numpy
restatement of the same algorithm, and its tangents against the complex-step derivative of the
numpy restatement with the Recfast steps replayed (CPU)."""
import warnings

import numpy as np
import pytest

from discoeb_b200 import _abi
from discoeb_b200.background import evolve_background, native_background
from discoeb_b200.gradients import ODE_DIRECTIONS, cosmology_prologue, param_dots, theta_to_params
from discoeb_b200.spline import spline_interpolation
from discoeb_b200.workloads import cosmo_params, sample_thetas

L = dict(lmaxg=12, lmaxgp=12, lmaxr=17, lmaxnu=17, nqmax=5)


def _numpy_bg(p, num_thermo=256, trace=None):
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        return evolve_background(param=p, num_thermo=num_thermo, backend="numpy", trace=trace)


def _max_rel(a, b):
    """max |a - b| / max |b| over the finite entries (non-finite entries must coincide)"""
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    fa, fb = np.isfinite(a), np.isfinite(b)
    if not np.array_equal(fa, fb) or not np.array_equal(a[~fa], b[~fb], equal_nan=True):
        return np.inf
    if not fb.any():
        return 0.0
    return float(np.max(np.abs(a[fb] - b[fb])) / max(np.max(np.abs(b[fb])), 1e-300))


def _compare(nat, ref):
    """max-normalised differences of every float field and spline table of two backgrounds"""
    assert set(nat) == set(ref)
    out = {}
    for k, v in ref.items():
        if isinstance(v, spline_interpolation):
            for f in ("x", "y", "S"):
                out[k + "." + f] = _max_rel(getattr(nat[k], f), getattr(v, f))
        elif np.asarray(v).dtype.kind == "f":
            out[k] = _max_rel(nat[k], v)
    return out


@pytest.mark.parametrize("m_nu,num_thermo", [(0.0, 256), (0.06, 256), (0.06, 1024)])
def test_native_background_matches_numpy_restatement(m_nu, num_thermo):
    p = cosmo_params(m_nu=m_nu, w0=-0.95, wa=0.1)
    trace = {}
    ref = _numpy_bg(p, num_thermo, trace)
    nat = evolve_background(param=p, num_thermo=num_thermo)
    diffs = _compare(nat, ref)
    # the same branches and the same GRK4A step sequence in every Recfast interval
    buf, _ = native_background(p, num_thermo)
    lay, _ = _abi.background_layout(num_thermo)
    np.testing.assert_array_equal(buf[lay["t:rec_case"]], trace["case"])
    np.testing.assert_array_equal(buf[lay["t:rec_steps"]], [len(s) for s in trace["steps"]])
    # values agree to rounding (knot second derivatives amplify it by 1/h^2).  xeprime_recf is left
    # out: in the hydrogen-Saha intervals the reference's closed form for dx_H/dz is the difference
    # of two terms of ~1e14 that cancel to rounding (the derivative of x_H = 1 - 3e-7), so its
    # value there is one ulp of those terms in either implementation
    diffs.pop("xeprime_recf")
    # the same formula's x_H = 0.5 (sqrt(r^2 + 4 r) - r) itself cancels for large r: the x_e tables
    # agree to 1e-6 of their scale (their knot second derivatives at 1024 knots: ~4e-7)
    xe_fields = {k: v for k, v in diffs.items() if k.startswith("xe")}
    worst = max(xe_fields.items(), key=lambda kv: kv[1])
    assert worst[1] < 1e-6, worst
    worst = max(((k, v) for k, v in diffs.items() if k not in xe_fields), key=lambda kv: kv[1])
    assert worst[1] < 1e-9, worst
    for k in ("grhom", "OmegaDE", "taumin", "taumax", "tau0", "amnu"):
        assert nat[k] == pytest.approx(ref[k], rel=1e-13, abs=0.0), k


def test_native_background_box_cosmologies():
    """Cosmologies of the uneven-batch box: identical Recfast branches and step counts; values to
    1e-4 (the Saha x_H formula of the reference cancels catastrophically just before hydrogen
    recombination, so a last-bit difference of exp/log between libm and numpy moves x_H there by
    ~1e-10 and x_He in the following intervals by up to ~1e-5)."""
    for theta in sample_thetas(3, seed=3):
        p = theta_to_params(theta)
        trace = {}
        ref = _numpy_bg(p, 256, trace)
        buf, _ = native_background(p)
        lay, _ = _abi.background_layout(256)
        np.testing.assert_array_equal(buf[lay["t:rec_case"]], trace["case"])
        np.testing.assert_array_equal(buf[lay["t:rec_steps"]], [len(s) for s in trace["steps"]])
        for nm in ("tau", "xe", "cs2", "Tm", "gvis", "optical_depth"):
            assert _max_rel(buf[lay["t:" + nm]], ref[nm]) < 1e-4, nm
        np.testing.assert_allclose(buf[lay["t:tau"]], ref["tau"], rtol=1e-12)


def test_native_background_rejects_bad_sizes():
    with pytest.raises(ValueError):
        native_background(cosmo_params(), num_thermo=16)
    lib = _abi.lib()
    assert lib.discoeb_background_size(16) == -1
    assert lib.discoeb_background_size(256) == _abi.background_layout(256)[1]


def test_native_tangents_match_complex_step_of_numpy_restatement():
    theta = dict(omega_c=0.12, omega_b=0.0224, h=0.674, n_s=0.965, ln10As=np.log(21.0), w0=-0.9, wa=0.05, m_nu=0.06)
    ks, aout = np.geomspace(1e-4, 10.0, 16), np.array([1 / 3, 0.5, 2 / 3, 1.0])
    nat = cosmology_prologue(theta, aout, ks, L)
    ref = cosmology_prologue(theta, aout, ks, L, host_backend="numpy", host_threads=1)
    for k in ("tau_out", "tau_start", "y0"):
        np.testing.assert_allclose(nat[k], ref[k], rtol=1e-12)
    y0_scale = np.abs(ref["y0"]).max(axis=0)
    for di, name in enumerate(ODE_DIRECTIONS):
        a, b = nat["tans"][di], ref["tans"][di]
        for f, v in b["scalars"].items():
            assert a["scalars"][f] == pytest.approx(v, rel=1e-9, abs=1e-14 * (abs(v) + 1.0)), (name, f)
        np.testing.assert_allclose(a["tau_out"], b["tau_out"], rtol=1e-9, err_msg=name)
        # the numpy path differentiates Recfast's Jacobian and the Saha He II slope by central
        # differences (relative steps 1e-7 and 1e-6) where forward mode is exact, and both go
        # through the reference's cancelling Saha x_H formula: tables agree to 1e-4 of their scale
        for short, (yy, SS) in b["tables"].items():
            assert _max_rel(a["tables"][short][0], yy) < 1e-4, (name, short)
            assert _max_rel(a["tables"][short][1], SS) < 1e-4, (name, short)
        assert np.all(np.abs(a["y0"] - b["y0"]) <= 1e-9 * y0_scale + 1e-9 * np.abs(b["y0"])), name


def test_overlapped_prologue_equals_one_background_call():
    """The native prologue takes the values from a value-only call while the tangent passes run
    on a helper thread: the result equals the prologue built from one call's buffers, bit for bit."""
    theta = dict(omega_c=0.118, omega_b=0.0221, h=0.69, n_s=0.965, ln10As=np.log(21.0), w0=-0.95, wa=-0.1, m_nu=0.1)
    ks, aout = np.geomspace(1e-4, 5.0, 24), np.array([0.5, 1.0])
    p = theta_to_params(theta)
    one = native_background(p, 256, param_dots(theta, ODE_DIRECTIONS))
    a = cosmology_prologue(theta, aout, ks, L)
    b = cosmology_prologue(theta, aout, ks, L, buffers=one)
    for k in ("tau_out", "tau_start", "y0", "sw"):
        np.testing.assert_array_equal(a[k], b[k])
    for ta, tb in zip(a["tans"], b["tans"]):
        assert ta["scalars"] == tb["scalars"]
        np.testing.assert_array_equal(ta["tau_out"], tb["tau_out"])
        np.testing.assert_array_equal(ta["y0"], tb["y0"])
        for short, (yy, SS) in tb["tables"].items():
            np.testing.assert_array_equal(ta["tables"][short][0], yy)
            np.testing.assert_array_equal(ta["tables"][short][1], SS)


@pytest.mark.parametrize("name", ["h", "w0", "m_nu"])
def test_native_tangents_match_central_differences_of_smooth_parts(name):
    """Scalars, conformal times and the neutrino tables do not go through Recfast's branches:
    there the tangent is the derivative of a smooth function, checked by central differences."""
    theta = dict(omega_c=0.12, omega_b=0.0224, h=0.674, n_s=0.965, ln10As=np.log(21.0), w0=-0.9, wa=0.05, m_nu=0.06)
    buf, dots = native_background(theta_to_params(theta), 256, param_dots(theta, [name]))
    lay, _ = _abi.background_layout(256)
    eps = 1e-5 * abs(theta[name])
    side = []
    for sgn in (1, -1):
        th = dict(theta)
        th[name] += sgn * eps
        side.append(native_background(theta_to_params(th), 256)[0])
    fd = (side[0] - side[1]) / (2 * eps)
    d = dots[0]
    for nm in ("grhom", "OmegaDE", "amnu", "taumax", "tau0", "Omegamnu"):
        i = lay["s:" + nm]
        assert d[i] == pytest.approx(fd[i], rel=1e-6, abs=1e-12 * abs(buf[i]) / eps), nm
    for key in ("n:logrhonu_y", "n:logpnu_y"):
        np.testing.assert_allclose(d[lay[key]], fd[lay[key]], rtol=1e-6, atol=1e-9 * np.abs(fd[lay[key]]).max() + 1e-14)
    # tau at the Recfast knots: an integral of 1/(da/dtau) (smooth in the parameters)
    np.testing.assert_allclose(d[lay["t:tau"]], fd[lay["t:tau"]], rtol=1e-6, atol=1e-8 * np.abs(fd[lay["t:tau"]]).max())


def test_background_batch_entry_validates_arguments():
    """The device entry rejects bad sizes and workspaces before it touches a GPU (every call below
    returns at its argument checks; the pointer values are never dereferenced)."""
    lib = _abi.lib()
    N = 256
    _, size = _abi.background_layout(N)
    work = 2 * max(N, _abi.NU_KNOTS) + 6 * N
    per_fw = (16 * (size + work) + 8 * (N + 1) + 255) // 256 * 256
    per_d = (8 * (size + work) + 8 * (N + 1) + 255) // 256 * 256
    assert lib.discoeb_background_batch_workspace_bytes(4, 6, N) == 4 * 6 * per_fw
    assert lib.discoeb_background_batch_workspace_bytes(4, 0, N) == 4 * per_d
    for args in ((0, 6, N), (4, -1, N), (4, 6, 16)):
        assert lib.discoeb_background_batch_workspace_bytes(*args) == -1
    ws = lib.discoeb_background_batch_workspace_bytes(4, 0, N)
    fake = 0x10000  # never dereferenced: each call fails its checks first
    assert lib.discoeb_background_batch(None, None, 4, 0, N, fake, ws, fake, None, None) == -1
    assert lib.discoeb_background_batch(fake, None, 4, 0, N, fake + 8, ws, fake, None, None) == -1  # misaligned
    assert lib.discoeb_background_batch(fake, None, 4, 0, N, fake, ws - 1, fake, None, None) == -1  # too small
    assert lib.discoeb_background_batch(fake, None, 4, 2, N, fake, ws, fake, None, None) == -1  # no tangent arrays
