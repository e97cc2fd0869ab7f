"""discoeb_sources_noalloc against discoeb_sources.

The no-allocation entry serves callers that cannot allocate device memory (a framework that
owns the GPU's memory, a host loop where allocation is not allowed): it keeps its scratch in an
array the library holds on the GPU instead of a buffer from the caller.  Two calls in a row
through it, via the C ABI, must both reproduce the caller-scratch entry exactly (same kernels;
the shared array is written before it is read, so the first call leaves nothing that changes
the second).  Collected last, so that a run stopping at the first failure has run every other
test; it passes alone in a fresh process as well.
"""
import numpy as np
import pytest

from conftest import background

pytestmark = pytest.mark.gpu

L11 = dict(lmaxg=11, lmaxgp=11, lmaxr=11, lmaxnu=8, nqmax=3)


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("no CUDA device: the -m gpu tests need a GPU")
    return torch


def test_noalloc_sources_equal_caller_scratch_twice(torch_cuda):
    from discoeb_b200.cmb import cmb_aexp_out, compute_sources
    from discoeb_b200.perturbations import solve_modes
    bg = background("disco_notebook", 1024)
    a = cmb_aexp_out()
    tau = bg["tau_of_a_spline"].evaluate(a)
    ks = np.geomspace(1e-3, 0.3, 10)
    y = solve_modes(param=bg, kmodes=ks, tau_out=tau, rtol=1e-4, atol=1e-4, pcoeff=0.25, icoeff=0.8, dcoeff=0.0,
                    factormax=20.0, factormin=0.3, max_steps=4096, return_full=True, as_tensor=True, **L11)
    ref = compute_sources(param=bg, yout=y, kmodes=ks, aexp_out=a, **L11)
    for _ in range(2):
        got = compute_sources(param=bg, yout=y, kmodes=ks, aexp_out=a, no_alloc=True, **L11)
        for name in ("S", "S1", "S2", "alphaprime", "polarization_term"):
            np.testing.assert_array_equal(got[name].cpu().numpy(), ref[name].cpu().numpy())
