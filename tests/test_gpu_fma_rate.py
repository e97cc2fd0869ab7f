"""discoeb_fma_rate (the FP64 FMA throughput probe behind the bench's roofline denominator) does
the work it counts: every chain's end value against the closed form of a <- a b + c (GPU)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_fma_rate_chains_end_at_the_closed_form():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("no CUDA device: the -m gpu tests need a GPU")
    from discoeb_b200 import _abi
    lib = _abi.lib()
    n = int(lib.discoeb_fma_rate_threads())
    assert n > 0 and n % 256 == 0
    out = torch.empty(n, dtype=torch.float64, device="cuda")
    flops = ctypes.c_double(0.0)
    iters = 1000
    assert lib.discoeb_fma_rate(iters, out.data_ptr(), n, ctypes.byref(flops), None) == 0
    assert lib.discoeb_fma_rate(iters, out.data_ptr(), n - 1, ctypes.byref(flops), None) == -1
    torch.cuda.synchronize()
    assert flops.value == 2.0 * 8 * iters * n
    b, c = 0.9999999, 1e-7
    tid = np.arange(n)
    fixed = c / (1.0 - b)
    a0 = 1e-3 * (tid % 97)[:, None] + np.arange(8)[None, :]
    expect = (b**iters * (a0 - fixed) + fixed).sum(axis=1)
    np.testing.assert_allclose(out.cpu().numpy(), expect, rtol=1e-9)
