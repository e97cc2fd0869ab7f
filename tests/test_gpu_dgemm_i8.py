"""The FP64 product on the int8 tensor cores (discoeb_dgemm_i8, tcgen05.mma kind::i8) against
numpy's FP64 product (GPU).

Exact cases: integer operands whose digits are the integers themselves give the exact integer
product.  General cases: the error stays within the splitting's bound
2^(1-7 slices) (max_k |A_ik| sum_k |B_jk| + sum_k |A_ik| max_k |B_jk|) plus FP64 rounding."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("no CUDA device: the -m gpu tests need a GPU")
    return torch


def _bound(A, B, slices):
    aA, aB = np.abs(A), np.abs(B)
    split = 2.0 ** (1 - 7 * slices) * (aA.max(axis=1)[:, None] * aB.sum(axis=1)[None, :] +
                                       aA.sum(axis=1)[:, None] * aB.max(axis=1)[None, :])
    return 2.0 * split + 8 * 2.2e-16 * (aA @ aB.T)


@pytest.mark.parametrize("slices,split", [(1, 1), (2, 3)])
def test_gpu_dgemm_i8_integers_exact(torch_cuda, slices, split):
    from discoeb_b200.cmb import dgemm_i8
    rng = np.random.default_rng(1)
    A = rng.integers(-100, 101, size=(300, 1000)).astype(np.float64)
    B = rng.integers(-100, 101, size=(260, 1000)).astype(np.float64)
    C = dgemm_i8(A, B, slices=slices, split=split).cpu().numpy()
    want = (A.astype(np.int64) @ B.astype(np.int64).T).astype(np.float64)
    np.testing.assert_array_equal(C, want)


@pytest.mark.parametrize("slices", [6, 7, 8])
def test_gpu_dgemm_i8_within_splitting_bound(torch_cuda, slices):
    from discoeb_b200.cmb import dgemm_i8
    rng = np.random.default_rng(slices)
    m, n, k = 513, 300, 2000          # no dimension a multiple of the 256 x 256 x 128 tiles
    A = rng.standard_normal((m, k)) * np.exp(rng.uniform(-7, 7, m))[:, None] * np.exp(-np.arange(k) / 400.0)
    B = rng.standard_normal((n, k)) * np.exp(rng.uniform(-7, 7, n))[:, None] * (1 + np.arange(k)) ** -0.8
    want = A @ B.T
    bound = _bound(A, B, slices)
    for split in (1, 2, 0):
        C = dgemm_i8(A, B, slices=slices, split=split).cpu().numpy()
        assert np.all(np.abs(C - want) <= bound), (slices, split, float(np.max(np.abs(C - want) / bound)))


def test_gpu_dgemm_i8_line_of_sight_shape(torch_cuda):
    """operands shaped like the frequency sum: a row of decaying complex coefficients (interleaved
    re, im) against M_l(p)-like rows spanning decades; slices 7 reach ~1e-12 of each row's scale"""
    from discoeb_b200.cmb import dgemm_i8
    rng = np.random.default_rng(7)
    nf = 1025
    eta = np.arange(nf) * 0.8
    ck = (rng.standard_normal((96, nf)) + 1j * rng.standard_normal((96, nf))) * np.exp(-eta / 60.0)[None, :] \
        * np.exp(1j * np.outer(np.log(np.geomspace(1e-4, 0.5, 96)), eta))
    ells = np.arange(0, 600, 3)
    Mq = (1.0 + (eta[None, :] / (1.0 + ells[:, None] / 2.0)) ** 2) ** -0.8 * np.exp(1j * eta[None, :] * 0.37) \
        / (1.0 + ells[:, None]) ** 1.6
    A = np.empty((96, 2 * nf)); A[:, 0::2], A[:, 1::2] = ck.real, ck.imag
    B = np.empty((len(ells), 2 * nf)); B[:, 0::2], B[:, 1::2] = 2 * Mq.real, -2 * Mq.imag
    want = A @ B.T
    C = dgemm_i8(A, B, slices=7).cpu().numpy()
    assert np.all(np.abs(C - want) <= _bound(A, B, 7))
    rowmax = np.abs(want).max(axis=1, keepdims=True)
    assert np.max(np.abs(C - want) / rowmax) < 1e-11


def test_gpu_dgemm_i8_nonfinite_row(torch_cuda):
    from discoeb_b200.cmb import dgemm_i8
    rng = np.random.default_rng(3)
    A = rng.standard_normal((40, 300))
    B = rng.standard_normal((50, 300))
    A[5, 17] = np.nan
    B[9, 3] = np.inf
    C = dgemm_i8(A, B, slices=7).cpu().numpy()
    assert np.isnan(C[5]).all() and np.isnan(C[:, 9]).all()
    ok = np.ones_like(C, dtype=bool)
    ok[5] = False
    ok[:, 9] = False
    want = A @ B.T
    assert np.all(np.abs(C - want)[ok] <= _bound(np.nan_to_num(A), np.nan_to_num(B), 7)[ok])


def test_gpu_dgemm_i8_arguments(torch_cuda):
    from discoeb_b200 import _abi
    lib = _abi.lib()
    assert lib.discoeb_dgemm_i8_workspace_bytes(0, 4, 4, 7, 0) < 0
    assert lib.discoeb_dgemm_i8_workspace_bytes(4, 4, 4, 9, 0) < 0
    assert lib.discoeb_dgemm_i8_workspace_bytes(4, 4, 4, 7, 0) > 0
    # a workspace one byte short is rejected before any launch
    nb = lib.discoeb_dgemm_i8_workspace_bytes(4, 4, 4, 7, 1)
    assert lib.discoeb_dgemm_i8(4, 4, 4, 0, 4, 0, 0, 4, 0, 0, 4, 7, 1, 256, nb, None) != 0
    assert lib.discoeb_dgemm_i8(4, 4, 4, 0, 4, 2, 0, 4, 0, 0, 4, 7, 1, 256, nb, None) != 0


@pytest.mark.parametrize("trans_a,trans_b", [(True, False), (False, True), (True, True)])
def test_gpu_dgemm_i8_transposed_operands(torch_cuda, trans_a, trans_b):
    """operands stored K-major over their other index (the forward-mode line of sight contracts
    over the modes: G = Omega^T A)"""
    from discoeb_b200.cmb import dgemm_i8
    rng = np.random.default_rng(11)
    m, n, k = 300, 520, 777
    A = rng.standard_normal((m, k)) * np.exp(rng.uniform(-5, 5, m))[:, None]
    B = rng.standard_normal((n, k)) * np.exp(rng.uniform(-5, 5, n))[:, None]
    C = dgemm_i8(A.T.copy() if trans_a else A, B.T.copy() if trans_b else B, slices=7, trans_a=trans_a,
                 trans_b=trans_b).cpu().numpy()
    assert np.all(np.abs(C - A @ B.T) <= _bound(A, B, 7))
