import ctypes
import os
import subprocess
import sys
import warnings

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "disco-eb_b200"))
sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (run with -m gpu)")


@pytest.fixture(scope="session")
def golden():
    return dict(np.load(os.path.join(GOLDEN, "reference_golden.npz")))


_BG = {}


def background(name, num_thermo, backend="native"):
    """Cached evolve_background of a named cosmology."""
    from discoeb_b200.background import evolve_background
    from discoeb_b200.workloads import cosmo_params
    key = (name, num_thermo, backend)
    if key not in _BG:
        if name == "disco_notebook":
            p = {"Omegam": 0.3099, "Omegab": 0.0488911, "H0": 67.742, "n_s": 0.96822, "A_s": 2.1064e-09,
                 "mnu": 0.06, "Tcmb": 2.7255, "YHe": 0.248, "Neff": 2.046, "Nmnu": 1, "w_DE_0": -0.99,
                 "w_DE_a": 0.0, "cs2_DE": 1.0, "Omegak": 0.0, "k_p": 0.05}
        elif name == "lcdm_massless":
            p = cosmo_params()
        elif name == "lcdm_mnu":
            p = cosmo_params(m_nu=0.06)
        else:
            raise KeyError(name)
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")
            _BG[key] = evolve_background(param=p, num_thermo=num_thermo, backend=backend)
    return _BG[key]


@pytest.fixture(scope="session")
def shim(tmp_path_factory):
    """The device model and stepper headers compiled for one host thread (tests/cpu_model)."""
    from discoeb_b200 import _abi
    out = str(tmp_path_factory.mktemp("shim") / "model_shim.so")
    subprocess.run(["g++", "-O2", "-fPIC", "-shared", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                    "-I", os.path.join(ROOT, "disco-eb_b200", "csrc"), "-o", out,
                    os.path.join(ROOT, "tests", "cpu_model", "model_shim.cpp")], check=True)
    S = ctypes.CDLL(out)
    dp = ctypes.POINTER(ctypes.c_double)
    CP = ctypes.POINTER(_abi.DiscoebCosmo)
    CT = ctypes.POINTER(_abi.DiscoebControl)
    ip = ctypes.POINTER(ctypes.c_int)
    S.shim_rhs.argtypes = [CP, ctypes.c_double, dp, ctypes.c_double, ctypes.c_int, dp, dp]
    S.shim_jacobian.argtypes = [CP, ctypes.c_double, dp, ctypes.c_double, ctypes.c_int, dp, dp]
    S.shim_wsolve.argtypes = [CP, ctypes.c_double, dp, ctypes.c_double, ctypes.c_int, ctypes.c_double, dp, dp]
    S.shim_solve_mode.argtypes = [CP, CT, ctypes.c_double, ctypes.c_double, dp, dp, ctypes.c_int, dp, dp, ip]
    S.shim_wsolve_mixed.argtypes = S.shim_wsolve.argtypes
    S.shim_solve_mode_mixed.argtypes = S.shim_solve_mode.argtypes
    S.shim_solve_mode_tangent.argtypes = [CP, ctypes.c_void_p, CT, ctypes.c_double, ctypes.c_double, dp, dp, dp,
                                          ctypes.c_int, dp, dp, dp, ip, dp, ctypes.c_int]
    S.shim_replay.argtypes = [CP, ctypes.c_double, ctypes.c_double, dp, dp, ctypes.c_int, dp, dp]
    S.shim_solve_mode_tangent_records.argtypes = [CP, ctypes.c_void_p, CT, ctypes.c_double, ctypes.c_double, dp, dp,
                                                  dp, ctypes.c_int, dp, dp, ip]
    S.shim_output_tangent.argtypes = [CP, ctypes.c_void_p, ctypes.c_double, ctypes.c_double, dp, dp, dp, dp, dp, dp]
    S.shim_projected_output_tangent.argtypes = [CP, ctypes.c_void_p, ctypes.c_double, ctypes.c_double, dp, dp, dp, dp]
    return S
