"""Observables of the linear power spectrum on the GPU.

The reference's ``get_xi_from_P``, ``get_power_smoothed``, ``power_Kaiser`` and
``power_multipoles`` (``src/discoeb/perturbations.py:1409-1564``, with ``savgol_filter`` of
``src/discoeb/util.py:291-327``), with the same keyword arguments, computed by the library's
kernels (``discoeb_power_amplitudes``, ``discoeb_savgol_log_power``, ``discoeb_power_kaiser``,
``discoeb_power_multipoles``, ``discoeb_xi_from_power``).  Inputs are numpy arrays or torch
tensors; results are numpy arrays, or torch tensors on the device when the main input is a torch
tensor.  The GPU is required.
"""
from __future__ import annotations

import numpy as np

from . import _abi


def _torch():
    import torch
    return torch


def _device(x, device):
    torch = _torch()
    if device is not None:
        return torch.device(device)
    if isinstance(x, torch.Tensor) and x.is_cuda:
        return x.device
    if not torch.cuda.is_available():
        raise RuntimeError("discoeb_b200 needs a CUDA device (there is no CPU path)")
    return torch.device("cuda", torch.cuda.current_device())


def _on(x, device):
    torch = _torch()
    if isinstance(x, torch.Tensor):
        return x.to(device=device, dtype=torch.float64).contiguous()
    return torch.as_tensor(np.ascontiguousarray(x, dtype=np.float64), device=device)


def _ret(t, as_torch):
    return t if as_torch else t.cpu().numpy()


def _stream(device):
    return _torch().cuda.current_stream(device).cuda_stream


def _check(rc, name):
    if rc != 0:
        raise RuntimeError(f"{name} failed with code {rc}")


def savgol_coeffs(window_length, polyorder):
    """Savitzky-Golay filter coefficients as util.py:291-327 computes them: the minimum-norm
    least-squares solution of A c = e_0 with A[o, j] = x_j^o (host, a (polyorder+1) x window
    system)."""
    halflen, rem = divmod(int(window_length), 2)
    pos = halflen - 0.5 if rem == 0 else halflen
    x = np.arange(-pos, window_length - pos, dtype=float)[::-1]
    A = x ** np.arange(polyorder + 1).reshape(-1, 1)
    Y = np.zeros(polyorder + 1)
    Y[0] = 1.0
    return np.linalg.lstsq(A, Y, rcond=None)[0]


def _fields(y, kmodes, param, idx, squared, device):
    """amplitudes (squared=0) or power (squared=1) of output field ``idx`` on the device"""
    torch = _torch()
    yy = _on(y, device)
    if yy.dim() != 2:
        raise ValueError("y must be [num_k, n_fields] (the outputs at one time)")
    k = _on(kmodes, device)
    n = k.shape[0]
    out = torch.empty(n, dtype=torch.float64, device=device)
    rc = _abi.lib().discoeb_power_amplitudes(n, k.data_ptr(), yy.data_ptr(), yy.shape[1], int(idx),
                                             float(param["A_s"]), float(param["n_s"]), float(param["k_p"]),
                                             int(squared), out.data_ptr(), _stream(device))
    _check(rc, "discoeb_power_amplitudes")
    return out


def _window_length(k, dlogk):
    kk = np.asarray(k.detach().cpu() if hasattr(k, "detach") else k, dtype=np.float64)
    wl = int(round(dlogk / (np.log(kk[1]) - np.log(kk[0]))))
    return wl + (wl + 1) % 2


def get_power_smoothed(*, k, y, dlogk, idx, param, device=None):
    """Savitzky-Golay (cubic) smoothed power spectrum in log k (perturbations.py:1471-1493)."""
    torch = _torch()
    as_torch = isinstance(y, torch.Tensor)
    device = _device(y, device)
    wl = _window_length(k, dlogk)
    P = _fields(y, k, param, idx, 1, device)
    c = torch.as_tensor(savgol_coeffs(wl, 3), device=device)
    out = torch.empty_like(P)
    rc = _abi.lib().discoeb_savgol_log_power(P.shape[0], P.data_ptr(), wl, c.data_ptr(), out.data_ptr(),
                                             _stream(device))
    _check(rc, "discoeb_savgol_log_power")
    return _ret(out, as_torch)


def power_Kaiser(*, y, kmodes, bias, mu_sampling=True, smooth_dlogk=None, nmu, param, device=None):
    """Anisotropic (Kaiser) spectrum P(k, mu) [num_k, nmu] and the mu samples
    (perturbations.py:1495-1524)."""
    torch = _torch()
    as_torch = isinstance(y, torch.Tensor)
    device = _device(y, device)
    mu = np.linspace(-1, 1, nmu) if mu_sampling else np.cos(np.linspace(0, np.pi, nmu))
    if smooth_dlogk is None:
        delta = _fields(y, kmodes, param, 4, 0, device)
        theta = _fields(y, kmodes, param, 5, 0, device)
    else:
        delta = torch.sqrt(_on(get_power_smoothed(k=kmodes, y=y, dlogk=smooth_dlogk, idx=4, param=param,
                                                  device=device), device))
        theta = -torch.sqrt(_on(get_power_smoothed(k=kmodes, y=y, dlogk=smooth_dlogk, idx=5, param=param,
                                                   device=device), device))
    mu_d = torch.as_tensor(mu, device=device)
    n = delta.shape[0]
    out = torch.empty((n, nmu), dtype=torch.float64, device=device)
    rc = _abi.lib().discoeb_power_kaiser(n, delta.data_ptr(), theta.data_ptr(), float(bias), int(nmu), mu_d.data_ptr(),
                                         out.data_ptr(), _stream(device))
    _check(rc, "discoeb_power_kaiser")
    return _ret(out, as_torch), (mu_d if as_torch else mu)


def power_multipoles(*, y, kmodes, b, param, device=None):
    """Monopole, quadrupole and hexadecapole of the Kaiser spectrum (perturbations.py:1528-1564)."""
    torch = _torch()
    as_torch = isinstance(y, torch.Tensor)
    device = _device(y, device)
    delta = _fields(y, kmodes, param, 4, 0, device)
    theta = _fields(y, kmodes, param, 5, 0, device)
    n = delta.shape[0]
    P = torch.empty((3, n), dtype=torch.float64, device=device)
    rc = _abi.lib().discoeb_power_multipoles(n, delta.data_ptr(), theta.data_ptr(), float(b), P[0].data_ptr(),
                                             P[1].data_ptr(), P[2].data_ptr(), _stream(device))
    _check(rc, "discoeb_power_multipoles")
    return tuple(_ret(P[i], as_torch) for i in range(3))


def get_xi_from_P(*, k, Pk, N=None, ell=0, device=None):
    """Correlation function multipole xi_l(r) from P(k) on log-spaced k by FFTLog
    (perturbations.py:1409-1442); returns (xi, r) in increasing r.  len(k) must be even."""
    torch = _torch()
    as_torch = isinstance(Pk, torch.Tensor)
    device = _device(Pk, device)
    kk, PP = _on(k, device), _on(Pk, device)
    n = kk.shape[0]
    if n % 2 or n < 2 or PP.shape[0] != n:
        raise ValueError("get_xi_from_P needs an even number of log-spaced k values and P(k) of the same length")
    lib = _abi.lib()
    wsb = lib.discoeb_xi_workspace_bytes(n)
    if wsb < 0:
        raise RuntimeError("discoeb_xi_workspace_bytes failed")
    ws = torch.empty(int(wsb) + 256, dtype=torch.uint8, device=device)
    base = (ws.data_ptr() + 255) & ~255
    xi = torch.empty(n, dtype=torch.float64, device=device)
    r = torch.empty(n, dtype=torch.float64, device=device)
    rc = lib.discoeb_xi_from_power(n, kk.data_ptr(), PP.data_ptr(), int(ell), base, int(wsb), xi.data_ptr(),
                                   r.data_ptr(), _stream(device))
    _check(rc, "discoeb_xi_from_power")
    return _ret(xi, as_torch), _ret(r, as_torch)
