"""One cosmology's modes spread over two ranks (gloo process group, both ranks on the one GPU this
test has; each rank's kernels run independently of the other's, the ranks meet only in the
CPU-side collectives): the gathered P(k) and Jacobian equal a single-process call, and C_l from
per-rank partial integrals equals the single-process chain on the modes' own k grid."""
import math
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

THETA = dict(omega_c=0.120, omega_b=0.0224, h=0.674, n_s=0.965, ln10As=math.log(21.0), w0=-0.9, wa=0.1, m_nu=0.06)
L65 = dict(lmaxg=12, lmaxgp=12, lmaxr=17, lmaxnu=3, nqmax=3)
PK = dict(aexp_out=(0.5, 1.0), kmin=1e-3, kmax=1.0, num_k=9, rtol=1e-5, atol=1e-8, **L65)
CMB = dict(ellmax=300, nmodes=24, n_fftlog=4096, spectra=("TT", "TE", "EE"))
PARAM = {"Omegam": 0.3099, "Omegab": 0.0488911, "H0": 67.742, "n_s": 0.96822, "A_s": 2.1064e-09, "mnu": 0.06,
         "Tcmb": 2.7255, "YHe": 0.248, "Neff": 2.046, "Nmnu": 1, "w_DE_0": -0.99, "w_DE_a": 0.0, "cs2_DE": 1.0,
         "Omegak": 0.0, "k_p": 0.05}


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import sys
    import warnings
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "disco-eb_b200"))
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      LOCAL_RANK=str(rank))
    try:
        from discoeb_b200 import replicas
        from discoeb_b200.cmb import compute_Cell_sharded
        from discoeb_b200.gradients import power_spectrum_jacobian_sharded
        _, _, dist = replicas.init("gloo", timeout_s=120)
        k, P, J = power_spectrum_jacobian_sharded(THETA, dist=dist, **PK)
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")
            cells, _ = compute_Cell_sharded(PARAM, dist=dist, **CMB)
        replicas.finish(dist)
        out.put((rank, k, P, J, {n: c for n, c in cells.items()}, None))
    except Exception as e:  # report instead of hanging the parent
        out.put((rank, None, None, None, None, repr(e)))


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("no CUDA device: the -m gpu tests need a GPU")
    return torch


def test_gpu_two_ranks_gather_power_and_reduce_cell(torch_cuda):
    import multiprocessing as mp
    import warnings
    from discoeb_b200.cmb import compute_Cell_spectrum_from_cosmo_params
    from discoeb_b200.gradients import power_spectrum_jacobian
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=600) for _ in procs), key=lambda r: r[0])
    for p in procs:
        p.join(timeout=120)
    assert all(r[5] is None for r in res), [r[5] for r in res]
    assert all(p.exitcode == 0 for p in procs)
    k1, P1, J1 = power_spectrum_jacobian(THETA, **PK)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        cells1, _ = compute_Cell_spectrum_from_cosmo_params(PARAM, n_k_dense=0, **CMB)
    for _, k, P, J, cells, _ in res:
        np.testing.assert_array_equal(k, k1)
        # each mode's solve is its own block: the shares reproduce the single call to rounding
        np.testing.assert_allclose(P, P1, rtol=1e-12, atol=0)
        np.testing.assert_allclose(J, J1, rtol=1e-10, atol=1e-12 * np.abs(J1).max())
        for name in CMB["spectra"]:
            scale = np.abs(cells1[name][2:]).max()
            np.testing.assert_allclose(cells[name][2:], cells1[name][2:], rtol=1e-10, atol=1e-12 * scale)
