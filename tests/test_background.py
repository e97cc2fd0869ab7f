"""Host background + Recfast restatement against the reference's golden data (CPU)."""
import numpy as np
import pytest

from conftest import background


@pytest.mark.parametrize("backend", ["native", "numpy"])
def test_background_matches_reference_golden(golden, backend):
    # tests/test_cmb/test_benchmark_evolve_background.csv: DISCO-Notebook cosmology, 1024 thermo points
    bg = background("disco_notebook", 1024, backend)
    assert bg["grhom"] == pytest.approx(float(golden["bg_grhom"][0]), rel=1e-14)
    tau = bg["tau_of_a_spline"].evaluate(golden["bg_a"])
    np.testing.assert_allclose(tau, golden["bg_tau"], rtol=1e-10)
    exp_xe = np.exp(bg["xe_of_loga_spline"].evaluate(np.log(golden["bg_a"])))
    np.testing.assert_allclose(exp_xe, golden["bg_exp_xe"], rtol=1e-9)


def test_spline_matches_reference_conventions():
    from discoeb_b200.spline import spline_interpolation
    x = np.linspace(0.0, 1.0, 11)
    y = np.sin(3 * x)
    s = spline_interpolation(x, y)
    assert s.S[0] == 0.0 and s.S[-1] == 0.0  # natural spline
    np.testing.assert_allclose(s.evaluate(x), y, rtol=0, atol=1e-15)
    # index = count(x < xn) - 1: a knot belongs to the interval on its left
    assert int(s._find_index(x[3])) == 2
    xs = np.linspace(0, 1, 1001)
    np.testing.assert_allclose(s.evaluate(xs), np.sin(3 * xs), atol=1e-3)  # natural end conditions
    u = spline_interpolation(x, y, uniform=True)
    np.testing.assert_allclose(u.evaluate(xs), s.evaluate(xs), rtol=0, atol=1e-14)
