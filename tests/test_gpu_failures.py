"""Failure detection on the device, without a GPU fault: a wait between the cooperating warps of a
mode that runs out of polls ends the mode with DISCOEB_ABORTED (the launch returns normally and
the context stays usable), and a NaN or an infinity in one cosmology's input table ends exactly
that cosmology's modes with DISCOEB_NONFINITE."""
import math
import warnings

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

L65 = dict(lmaxg=12, lmaxgp=12, lmaxr=17, lmaxnu=3, nqmax=3)
THETA = dict(omega_c=0.120, omega_b=0.0224, h=0.674, n_s=0.965, ln10As=math.log(21.0), w0=-0.9, wa=0.1, m_nu=0.06)


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("no CUDA device: the -m gpu tests need a GPU")
    return torch


def test_gpu_exhausted_wait_aborts_every_mode_and_the_context_survives(torch_cuda):
    torch = torch_cuda
    from discoeb_b200.gradients import JacobianProblem
    prob = JacobianProblem(THETA, aexp_out=(0.5, 1.0), kmin=1e-3, kmax=1.0, num_k=6, rtol=1e-5, atol=1e-8, **L65)
    prob.ctrl.max_polls = 1  # a tangent warp gives up after one poll of the forward's hand-over counter
    prob.launch()
    torch.cuda.synchronize()
    P, J, status, nsteps = prob.result(on_failure="ignore")
    assert (status == 6).all(), status  # DISCOEB_ABORTED
    assert np.isnan(J[:6]).any()
    # the same problem with the default budget runs normally afterwards on the same context
    prob.ctrl.max_polls = 0
    prob.launch()
    P, J, status, nsteps = prob.result()
    assert (status == 0).all() and np.isfinite(J).all()


def test_gpu_nonfinite_table_fails_only_its_cosmology(torch_cuda):
    from discoeb_b200.background import evolve_background
    from discoeb_b200.gradients import theta_to_params
    from discoeb_b200.perturbations import CosmologyBatch
    from discoeb_b200.workloads import sample_thetas
    thetas = sample_thetas(4, seed=5)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        bgs = [evolve_background(param=theta_to_params(t)) for t in thetas]
    ks = np.geomspace(1e-3, 1.0, 5)
    batch = CosmologyBatch(params=bgs, kmodes=ks, aexp_out=np.array([0.5, 1.0]), rtol=1e-5, atol=1e-8, **L65)
    # DeviceCosmo.tensors hold each table as rows x, y, S: poison the knot values of cosmology 1's
    # x_e table with NaN and those of cosmology 2's c_s^2 a table with +inf
    n_xe = bgs[1]["xe_of_loga_spline"].n
    batch.dcs[1].tensors[0].view(-1)[n_xe:2 * n_xe] = float("nan")
    n_cs = bgs[2]["cs2a_of_loga_spline"].n
    batch.dcs[2].tensors[1].view(-1)[n_cs:2 * n_cs] = float("inf")
    batch.launch()
    y, status, nsteps = batch.result(on_failure="ignore")
    assert (status[0] == 0).all() and (status[3] == 0).all(), status
    assert (status[1] == 2).all() and (status[2] == 2).all(), status  # DISCOEB_NONFINITE
    assert np.isfinite(y[[0, 3]]).all()
    assert np.isnan(y[[1, 2]]).all()  # outputs never reached are NaN
    # the poisoned modes stop at their first step instead of shrinking the step to underflow
    assert (nsteps[1] == 1).all() and (nsteps[2] == 1).all(), nsteps
