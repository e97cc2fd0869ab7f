"""Host-side logic of the package and the C ABI library surface (CPU, no GPU calls)."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT, background
from discoeb_b200 import _abi
from discoeb_b200 import perturbations as pert
from oracle import pyoracle as O

L = dict(lmaxg=12, lmaxgp=12, lmaxr=17, lmaxnu=17, nqmax=5)


def test_start_times_and_ics_match_oracle():
    bg = background("disco_notebook", 512)
    OP = O.OracleProblem(bg, **L)
    ks = np.geomspace(1e-5, 10.0, 23)
    ts = pert.determine_starting_time(param=bg, k=ks)
    np.testing.assert_allclose(ts, [OP.start_time(k) for k in ks], rtol=1e-12)
    y = pert.adiabatic_ics(tau=ts, param=bg, kmode=ks, **L)
    yo = np.stack([OP.ics(t, k) for t, k in zip(ts, ks)])
    np.testing.assert_allclose(y, yo, rtol=1e-12, atol=0)


def test_switch_times_match_oracle():
    bg = background("disco_notebook", 512)
    OP = O.OracleProblem(bg, **L)
    ks = np.geomspace(1e-4, 10.0, 17)
    sw = pert.approximation_switch_times(bg, ks)
    so = np.stack([OP.switch_times(k) for k in ks])
    np.testing.assert_allclose(sw[:, :2], so[:, :2], rtol=1e-9)
    assert np.isinf(sw[:, 2]).all()


def test_k_sampling_and_errors():
    bg = background("disco_notebook", 256)
    k = pert.k_sampling(bg, 1e-4, 1.0, 64, "camb")
    assert k.shape == (64,) and np.all(np.diff(k) > 0)
    with pytest.raises(ValueError):
        pert.k_sampling(bg, 1e-4, 1.0, 64, "nope")
    with pytest.raises(ValueError):
        pert.k_sampling({}, 1e-4, 1.0, 64, "camb")
    with pytest.raises(ValueError):
        pert.evolve_perturbations_batched(param=bg, aexp_out=[1.0], kmin=1e-4, kmax=1.0, num_k=10, batch_size=4)


def test_get_power_formula():
    p = {"A_s": 2.1e-9, "n_s": 0.965, "k_p": 0.05}
    k = np.array([0.01, 0.1])
    y = np.zeros((2, 1, 20))
    y[:, 0, 4] = [3.0, 4.0]
    P = pert.get_power(k=k, y=y[:, -1, :], idx=4, param=p)
    np.testing.assert_allclose(P, 2 * np.pi**2 * 2.1e-9 * (k / 0.05) ** -0.035 * k ** -3 * np.array([9.0, 16.0]))


def test_library_exports_every_declared_symbol():
    path = os.path.join(ROOT, "disco-eb_b200", "discoeb_b200", _abi.LIB_NAME)
    if not os.path.exists(path):
        subprocess.run(["python", os.path.join(ROOT, "disco-eb_b200", "build.py")], check=True)
    declared = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", h)).read()
            declared |= set(re.findall(r"^\s*(?:int32_t|int64_t|void|double)\s+(discoeb_\w+)\s*\(", txt, re.M))
    assert {"discoeb_fwd", "discoeb_rhs", "discoeb_nvar", "discoeb_abi_version", "discoeb_los_workspace_bytes",
            "discoeb_background", "discoeb_background_size", "discoeb_fma_rate", "discoeb_fma_rate_threads"} <= declared
    lib = ctypes.CDLL(path)
    for name in declared:
        assert hasattr(lib, name), name
    assert lib.discoeb_abi_version() == _abi.ABI_VERSION
    c = _abi.DiscoebCosmo()
    c.lmaxg, c.lmaxgp, c.lmaxr, c.lmaxnu, c.nqmax = 12, 12, 17, 17, 5
    lib.discoeb_nvar.restype = ctypes.c_int32
    assert lib.discoeb_nvar(ctypes.byref(c)) == 143


def test_fma_rate_entry_rejects_bad_arguments_before_any_launch():
    lib = _abi.lib()
    flops = ctypes.c_double(-1.0)
    # checked before the device is touched, so these run without a GPU
    assert lib.discoeb_fma_rate(0, 256, 1 << 20, ctypes.byref(flops), None) == -1
    assert lib.discoeb_fma_rate(10, None, 1 << 20, ctypes.byref(flops), None) == -1
    assert lib.discoeb_fma_rate(10, 256, 1 << 20, None, None) == -1
    assert flops.value == -1.0


def test_jvp_entries_reject_missing_outputs_before_any_launch():
    lib = _abi.lib()
    host = _abi.DiscoebCosmo()
    host.lmaxg, host.lmaxgp, host.lmaxr, host.lmaxnu, host.nqmax = 11, 11, 11, 8, 3
    ctrl = _abi.DiscoebControl(1e-4, 1e-4, 0.25, 0.8, 0.0, 20.0, 0.3, 2048, _abi.METHOD_RODAS5_STRUCTURED, 0, 0)
    fake = 4096  # never dereferenced: the argument checks return first
    for entry in (lib.discoeb_jvp, lib.discoeb_jvp_full):
        args = [fake, ctypes.byref(host), 1, None, fake, 6, ctypes.byref(ctrl), 8, fake, fake, fake, fake, fake, 4,
                fake, fake, fake, None, fake, fake, None]
        assert entry(*args) == -1  # no derivative output
        args[5] = 0
        assert entry(*args) == -1  # no direction


def test_line_of_sight_tangent_entry_rejects_bad_arguments_before_any_launch():
    lib = _abi.lib()
    f = lib.discoeb_los_cell_jvp
    fake = 4096  # never dereferenced: the argument checks return first
    t0d = (ctypes.c_double * 2)(0.0, 0.0)
    ok = [8, fake, 16, fake, fake, 1.0e4, 2, fake, fake, ctypes.addressof(t0d), 100, 256, 0, 0.96, 0.05, 4096, 1 << 30,
          fake, fake, None, None]
    bad = [(0, 1), (2, 2), (10, -1), (11, 1), (12, 1), (15, None), (6, -1)]  # sizes, workspace, n_dir
    for i, v in bad:
        args = list(ok)
        args[i] = v
        assert f(*args) == -1, (i, v)
    args = list(ok)
    args[8] = None  # directions without their source tangents
    assert f(*args) == -1
    args = list(ok)
    args[15] = 4097  # workspace not 256-byte aligned
    assert f(*args) == -1
    assert lib.discoeb_los_cell_jvp_workspace_bytes(1, 16, 100, 256, 0) == -1


def test_native_spline_recurrence_equals_the_reference_recurrence_bitwise():
    """spline_interpolation's knot second derivatives come from the library's host restatement of
    the reference's Thomas recurrence (spline_interpolation.py:19-75); the recurrence written out
    on numpy float64 scalars gives the same bits."""
    from discoeb_b200.spline import spline_interpolation

    def recurrence(x, y):
        n = len(y)
        S = np.zeros(n)
        m = n - 2
        if m <= 0:
            return S
        h = x[1:] - x[:-1]
        a, b, c = h[:-1], 2.0 * (h[:-1] + h[1:]), h[1:]
        d = 6.0 * ((y[2:] - y[1:-1]) / h[1:] - (y[1:-1] - y[:-2]) / h[:-1])
        cp, dp = np.zeros(m), np.zeros(m)
        cp[0], dp[0] = c[0] / b[0], d[0] / b[0]
        for i in range(1, m):
            den = b[i] - a[i] * cp[i - 1]
            cp[i] = c[i] / den if i < m - 1 else 0.0
            dp[i] = (d[i] - a[i] * dp[i - 1]) / den
        Si = np.zeros(m)
        Si[m - 1] = dp[m - 1]
        for i in range(m - 2, -1, -1):
            Si[i] = dp[i] - cp[i] * Si[i + 1]
        S[1:-1] = Si
        return S

    rng = np.random.default_rng(7)
    for n in (2, 3, 4, 17, 1024):
        x = np.sort(rng.uniform(-3.0, 10.0, n))
        y = np.exp(-x) + rng.normal(size=n) * 1e-3
        np.testing.assert_array_equal(spline_interpolation(x, y).S, recurrence(x, y))
    # complex (complex-step) data keeps the numpy recurrence, whose real part is the same spline
    x = np.sort(rng.uniform(0.0, 5.0, 64))
    y = np.sin(x)
    Sc = spline_interpolation(x, y + 1e-30j * np.cos(x)).S
    np.testing.assert_allclose(Sc.real, recurrence(x, y), rtol=1e-12, atol=1e-13)
    assert _abi.lib().discoeb_natural_spline_second(1, 0, 0, 0) == -1


def test_cell_jacobian_rejects_an_unknown_line_of_sight_mode():
    from discoeb_b200.cmb import compute_Cell_jacobian
    theta = dict(omega_c=0.12, omega_b=0.0224, h=0.674, n_s=0.965, ln10As=3.04, w0=-0.95, wa=0.0, m_nu=0.06)
    with pytest.raises(ValueError):
        compute_Cell_jacobian(theta, los="adjoint")


def test_sources_tangent_entry_rejects_bad_arguments_before_any_launch():
    lib = _abi.lib()
    host = _abi.DiscoebCosmo()
    host.lmaxg, host.lmaxgp, host.lmaxr, host.lmaxnu, host.nqmax = 11, 11, 11, 8, 3
    fake = 4096  # never dereferenced: the argument checks return first
    ok = [fake, ctypes.byref(host), fake, 1, 8, fake, 16, fake, fake, fake, fake, fake, fake, fake, fake, fake, None,
          None]
    for i, v in ((3, 0), (4, -1), (6, 2), (14, None), (15, None), (0, None)):
        args = list(ok)
        args[i] = v
        assert lib.discoeb_sources_jvp(*args) == -1, (i, v)


def test_noalloc_size_limit_is_the_same_in_c_and_python():
    # the no-allocation sources entry holds 2^20 points in its own array: one point more is refused
    # by the C entry before any device work (its pointers are never touched), and the Python
    # pre-check draws the line at the same place
    from discoeb_b200 import cmb
    lib = _abi.lib()
    host = _abi.DiscoebCosmo()
    assert cmb.NOALLOC_MAX_POINTS == 1 << 20
    assert lib.discoeb_sources_noalloc(None, ctypes.byref(host), 1025, None, 1024, None, None, None, None, None) == -1
    assert lib.discoeb_sources_noalloc(None, ctypes.byref(host), 1, None, (1 << 20) + 1, None, None, None, None,
                                       None) == -1
    cmb.noalloc_check(1024, 1024)
    cmb.noalloc_check(1, 1 << 20)
    with pytest.raises(ValueError):
        cmb.noalloc_check(1025, 1024)
    with pytest.raises(ValueError):
        cmb.noalloc_check(1, (1 << 20) + 1)


def test_sources_entries_refuse_grids_beyond_the_launch_limits():
    # one warp per (direction, mode, time) point: sizes whose grid would not fit are refused before
    # any launch (the pointers are never dereferenced)
    lib = _abi.lib()
    host = _abi.DiscoebCosmo()
    host.lmaxg, host.lmaxgp, host.lmaxr, host.lmaxnu, host.nqmax = 11, 11, 11, 8, 3
    fake = 4096
    big = 1 << 30
    assert lib.discoeb_sources_jvp(fake, ctypes.byref(host), fake, 8, big, fake, 16, fake, fake, fake, fake, fake,
                                   fake, fake, fake, fake, None, None) == -1
    assert lib.discoeb_sources(fake, ctypes.byref(host), big, fake, 64, fake, fake, fake, fake, fake, None) == -1


def test_struct_layout_matches_header():
    # the ctypes mirror must have the C layout: compile a tiny probe of offsetof/sizeof
    import tempfile
    src = r'''
#include <stddef.h>
#include <stdio.h>
#include "discoeb.h"
int main(void){printf("%zu %zu %zu %zu %zu %zu %d %d %d %d\n", sizeof(DiscoebCosmo), offsetof(DiscoebCosmo, q),
 offsetof(DiscoebCosmo, xe_loga), sizeof(DiscoebControl), offsetof(DiscoebControl, max_steps),
 sizeof(DiscoebCosmoParams), DISCOEB_BGS_COUNT, DISCOEB_BGN_COUNT, DISCOEB_BGT_COUNT, DISCOEB_NU_KNOTS);return 0;}
'''
    with tempfile.TemporaryDirectory() as d:
        open(os.path.join(d, "p.c"), "w").write(src)
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), "-o", os.path.join(d, "p"), os.path.join(d, "p.c")],
                       check=True)
        out = subprocess.run([os.path.join(d, "p")], capture_output=True, text=True, check=True).stdout.split()
    C, K = _abi.DiscoebCosmo, _abi.DiscoebControl
    assert [int(v) for v in out] == [ctypes.sizeof(C), C.q.offset, C.xe_loga.offset, ctypes.sizeof(K),
                                     K.max_steps.offset, ctypes.sizeof(_abi.DiscoebCosmoParams), len(_abi.BGS),
                                     len(_abi.BGN), len(_abi.BGT), _abi.NU_KNOTS]


def test_plain_c_caller_of_the_background_entry():
    """The C ABI from C: a program that includes discoeb.h and links the library gets the same
    background scalars and H0-derivatives as the Python layer (host entry; no GPU needed)."""
    import tempfile

    from discoeb_b200.background import native_background
    from discoeb_b200.workloads import cosmo_params
    libdir = os.path.join(ROOT, "disco-eb_b200", "discoeb_b200")
    if not os.path.exists(os.path.join(libdir, _abi.LIB_NAME)):
        subprocess.run(["python", os.path.join(ROOT, "disco-eb_b200", "build.py")], check=True)
    p = cosmo_params(m_nu=0.06, w0=-0.95, wa=0.1)
    with tempfile.TemporaryDirectory() as d:
        exe = os.path.join(d, "bg")
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), "-o", exe,
                        os.path.join(ROOT, "tests", "c_abi", "background_from_c.c"), "-L", libdir,
                        "-l:" + _abi.LIB_NAME, "-Wl,-rpath," + libdir], check=True)
        args = [repr(float(p[k])) for k in ("H0", "Omegab", "Omegam", "mnu", "w_DE_0", "w_DE_a")]
        txt = subprocess.run([exe, *args], capture_output=True, text=True, check=True).stdout.split()
    got = np.array([float(v) for v in txt]).reshape(-1, 2)
    buf, dots = native_background(p, 256, [{"H0": 1.0}])
    assert got.shape == (len(_abi.BGS), 2)
    np.testing.assert_array_equal(got[:, 0], buf[: len(_abi.BGS)])
    np.testing.assert_array_equal(got[:, 1], dots[0][: len(_abi.BGS)])


def test_fused_sources_entry_rejects_bad_arguments_before_any_launch():
    lib = _abi.lib()
    host = _abi.DiscoebCosmo()
    host.lmaxg, host.lmaxgp, host.lmaxr, host.lmaxnu, host.nqmax = 11, 11, 11, 8, 3
    ctrl = _abi.DiscoebControl(1e-4, 1e-4, 0.25, 0.8, 0.0, 20.0, 0.3, 2048, _abi.METHOD_RODAS5_STRUCTURED, 0, 0)
    fake = 4096  # never dereferenced: the argument checks return first
    ok = [fake, ctypes.byref(host), ctypes.byref(ctrl), 4, fake, fake, fake, fake, 16, fake, fake, None, fake, fake,
          fake, fake, None]
    for i, v in ((0, None), (3, -1), (8, 2), (12, None), (13, None), (14, None), (9, None)):
        args = list(ok)
        args[i] = v
        assert lib.discoeb_fwd_sources(*args) == -1, (i, v)
    bad = _abi.DiscoebControl(1e-4, 1e-4, 0.25, 0.8, 0.0, 20.0, 0.3, 2048, _abi.METHOD_RODAS5_STRUCTURED_MIXED, 0, 0)
    args = list(ok)
    args[2] = ctypes.byref(bad)
    assert lib.discoeb_fwd_sources(*args) == -3  # DISCOEB_EUNSUPPORTED


def test_int8_contraction_workspace_and_arguments_on_the_host():
    """discoeb_dgemm_i8's workspace arithmetic and argument checks (host code, no launch): digit
    planes of 256-row tiles x 128-byte K stages, the K ranges chosen for >= 4 waves of CTAs (148
    SMs assumed without a device), int32 level sums per K range and level"""
    lib = _abi.lib()
    tile = 256 * 128

    def planes(m, n, k, s):
        mt, nt, kst = -(-m // 256), -(-n // 256), -(-k // 128)
        return mt, nt, kst, s * (mt + nt) * kst * tile

    for (m, n, k, s, split) in [(8192, 2501, 16386, 7, 2), (300, 260, 1000, 1, 1), (513, 300, 2000, 6, 3)]:
        mt, nt, kst, pl = planes(m, n, k, s)
        got = lib.discoeb_dgemm_i8_workspace_bytes(m, n, k, s, split)
        levels = split * s * mt * 256 * nt * 256 * 4
        assert pl + levels <= got <= pl + levels + 8 * 256 + 8 * 12 * (mt + nt) * 256, (m, n, k, got)
    # the line-of-sight size without a split given: 320 tiles -> 2 K ranges (640 CTAs >= 4 x 148)
    assert lib.discoeb_dgemm_i8_workspace_bytes(8192, 2501, 16386, 7, 0) == \
        lib.discoeb_dgemm_i8_workspace_bytes(8192, 2501, 16386, 7, 2)
    for bad in [(0, 4, 4, 7, 0), (4, 0, 4, 7, 0), (4, 4, 0, 7, 0), (4, 4, 4, 0, 0), (4, 4, 4, 9, 0)]:
        assert lib.discoeb_dgemm_i8_workspace_bytes(*bad) < 0, bad
    nb = lib.discoeb_dgemm_i8_workspace_bytes(4, 4, 4, 7, 1)
    # null operands, a bad transpose flag, leading dimensions below the row length, a short or
    # unaligned workspace: all refused before any launch
    assert lib.discoeb_dgemm_i8(4, 4, 4, None, 4, 0, None, 4, 0, None, 4, 7, 1, 256, nb, None) != 0
    assert lib.discoeb_dgemm_i8(4, 4, 4, 256, 4, 2, 256, 4, 0, 256, 4, 7, 1, 256, nb, None) != 0
    assert lib.discoeb_dgemm_i8(4, 4, 4, 256, 3, 0, 256, 4, 0, 256, 4, 7, 1, 256, nb, None) != 0
    assert lib.discoeb_dgemm_i8(4, 4, 4, 256, 4, 0, 256, 4, 0, 256, 4, 7, 1, 256, nb - 1, None) != 0
    assert lib.discoeb_dgemm_i8(4, 4, 4, 256, 4, 0, 256, 4, 0, 256, 4, 7, 1, 264, nb, None) != 0
    assert lib.discoeb_set_los_contraction(2, 7) != 0 and lib.discoeb_set_los_contraction(1, 9) != 0
