"""The CPU oracle pinned against the reference's golden data and known answers (CPU)."""
import numpy as np
import pytest

from conftest import background
from oracle import pyoracle as O

AOUT_GOLDEN = np.concatenate([np.geomspace(3e-4, 5e-3, 256, endpoint=False), np.geomspace(5e-3, 1.0, 64)])


def test_oracle_final_states_match_reference_golden(golden):
    # tests/test_cmb/test_benchmark_evolve_perturbations_batched.csv was produced with
    # rtol = atol = 1e-4, 64 log-spaced modes in [1e-4, 1], lmax 11/11/11/8, nq 3.  A converged
    # oracle solve (rtol 1e-8, steps ending on every output) must reproduce its final states to
    # within that run's own integration error.
    bg = background("disco_notebook", 1024)
    ks = golden["pert_kmodes"][[0, 31, 63]]
    np.testing.assert_allclose(ks, np.geomspace(1e-4, 1.0, 64)[[0, 31, 63]], rtol=1e-12)
    y, k, st = O.evolve_perturbations(param=bg, aexp_out=AOUT_GOLDEN, kmin=0, kmax=0, num_k=0, rtol=1e-8, atol=1e-8,
                                      max_steps=100000, return_full=True, kmodes=ks, mode="clip")
    assert all(s[3] == 0 for s in st)
    sel = golden["pert_out_index"]
    for i, key in enumerate(("pert_y_k0", "pert_y_k31", "pert_y_k63")):
        g = golden[key]
        mine = y[i][sel]
        for v in (2, 3, 5):  # eta, delta_c, delta_b at a = 1
            assert mine[-1, v] == pytest.approx(g[-1, v], rel=2e-4), (key, v)
        # whole history: within the reference test's own tolerance (rtol 0.2) where the
        # reference's linear interpolation between its accepted steps is not dominant
        big = np.abs(g[:, 3]) > 1e-3 * np.abs(g[:, 3]).max()
        np.testing.assert_allclose(mine[big, 3], g[big, 3], rtol=0.2)


def test_oracle_reference_mode_reproduces_batched_golden(golden):
    # the reference's own semantics: batches of 16 modes sharing one step size, linear
    # interpolation to the outputs, switches evaluated per RHS call
    bg = background("disco_notebook", 1024)
    ks = np.geomspace(1e-4, 1.0, 64)
    y, k, st = O.evolve_perturbations(param=bg, aexp_out=AOUT_GOLDEN, kmin=0, kmax=0, num_k=0, rtol=1e-4, atol=1e-4,
                                      return_full=True, kmodes=ks[:32], mode="reference", batch_size=16)
    g = golden["pert_y_k0"]
    assert y[0][-1, 3] == pytest.approx(g[-1, 3], rel=1e-5)
    assert y[31][-1, 3] == pytest.approx(golden["pert_y_k31"][-1, 3], rel=1e-4)


def test_oracle_pk_matches_class(golden):
    # tests/test_perturbations.py:225-239: P_bc at a = 0.01 within 0.5% of CLASS, lmax 31, nq 5
    bg = background("disco_notebook", 1024)
    kc, pc = golden["class_k"], golden["class_pkbc"]
    m = (kc >= 1e-5) & (kc <= 1e2)
    kc, pc = kc[m][::24], pc[m][::24]
    y, k, st = O.evolve_perturbations(param=bg, aexp_out=[0.01], kmin=0, kmax=0, num_k=0, lmaxg=31, lmaxgp=31,
                                      lmaxr=31, lmaxnu=31, nqmax=5, rtol=1e-5, atol=1e-5, kmodes=kc, mode="clip",
                                      max_steps=20000)
    P = 2 * np.pi**2 * bg["A_s"] * (k / 0.05) ** (bg["n_s"] - 1) * k ** -3 * y[:, -1, 6] ** 2
    np.testing.assert_allclose(P, pc, rtol=5e-3)


def test_oracle_jacobian_matches_finite_differences():
    bg = background("disco_notebook", 256)
    OP = O.OracleProblem(bg, lmaxg=8, lmaxgp=8, lmaxr=8, lmaxnu=4, nqmax=3)
    k = 0.05
    ts = OP.start_time(k)
    y0 = OP.ics(ts, k)
    tout = bg["tau_of_a_spline"].evaluate(np.array([1e-3]))
    ys, st = OP.solve([k], ts, y0, tout, rtol=1e-6, atol=1e-9)
    y = ys[0, 0]
    tau = tout[0]
    J, dT = OP.jacobian(tau, y, k)
    n = OP.n
    for j in range(n):
        e = np.zeros(n)
        # rows >= 1 are linear in y[1:], so a floor on the step costs no accuracy; without it a
        # zero entry (theta_c in the synchronous gauge) gets a step at the rounding level
        h = 1e-6 * max(abs(y[j]), 1e-4)
        e[j] = h
        fd = (OP.rhs(tau, y + e, k) - OP.rhs(tau, y - e, k)) / (2 * h)
        np.testing.assert_allclose(J[:, j], fd, rtol=1e-5, atol=1e-6 * np.abs(J).max())
    h = 1e-6 * tau
    fd = (OP.rhs(tau + h, y, k) - OP.rhs(tau - h, y, k)) / (2 * h)
    np.testing.assert_allclose(dT, fd, rtol=1e-4, atol=1e-9 * np.abs(dT).max() + 1e-300)


def test_dark_energy_guard_is_the_lambda_limit():
    # w = -1 exactly gives NaN in the reference equations; the guarded solve equals the
    # w -> -1 limit of the unguarded equations
    from discoeb_b200.background import evolve_background
    from discoeb_b200.workloads import cosmo_params
    import warnings
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        bg1 = evolve_background(param=cosmo_params(w0=-1.0))
        bg2 = evolve_background(param=cosmo_params(w0=-1.0 + 1e-7))
    ks = np.geomspace(1e-3, 1.0, 4)
    kw = dict(aexp_out=[1.0], kmin=0, kmax=0, num_k=0, lmaxg=8, lmaxgp=8, lmaxr=8, lmaxnu=3, nqmax=3, rtol=1e-7,
              atol=1e-10, kmodes=ks, mode="clip")
    y0, _, _ = O.evolve_perturbations(param=bg1, de_guard_eps=0.0, **kw)
    assert not np.isfinite(y0[:, -1, 4]).all()  # the reference equations at w = -1
    y1, _, _ = O.evolve_perturbations(param=bg1, de_guard_eps=1e-9, **kw)
    y2, _, _ = O.evolve_perturbations(param=bg2, de_guard_eps=0.0, **kw)
    np.testing.assert_allclose(y1[:, -1, 4], y2[:, -1, 4], rtol=1e-5)
