"""Natural cubic spline tables (host side).

Restates ``spline_interpolation`` of the reference
(``src/discoeb/spline_interpolation.py:6-276``): knots ``x``, values ``y`` and the
second derivatives ``S`` at the knots from a natural-boundary tridiagonal (Thomas)
solve, plus cumulative interval integrals.  The three arrays ``(x, y, S)`` are the
table format the device kernels read: the CUDA path evaluates exactly the
polynomial of ``evaluate``/``derivative`` below, with the interval index chosen as
``count(x < x_new) - 1`` clipped to ``[0, n-2]`` (``_find_index``,
``spline_interpolation.py:132-145``), or ``floor((x_new - x0)/dx)`` for uniform
knot grids.
"""
from __future__ import annotations

import numpy as np


class spline_interpolation:
    """Natural cubic spline through ``(xin, yin)`` (reference class of the same name)."""

    def __init__(self, xin, yin, integrate_from_start: bool = True, uniform: bool = False):
        x = np.array(xin).ravel()
        x = x.astype(np.result_type(x.dtype, np.float64))
        y = np.array(yin).ravel()
        y = y.astype(np.result_type(y.dtype, np.float64))
        n = y.shape[0]
        if n < 2:
            raise ValueError("There must be at least two data points.")
        # forward-fill NaNs (spline_interpolation.py:33-40): y repeats the last
        # finite value, x grows geometrically by 1.01
        if np.isnan(np.real(y)).any() or np.isnan(np.real(x)).any():
            for i in range(n):
                prev_y = y[i - 1] if i > 0 else y[0]
                prev_x = x[i - 1] if i > 0 else x[0]
                if np.isnan(y[i]):
                    y[i] = prev_y
                if np.isnan(x[i]):
                    x[i] = prev_x * 1.01
        h = x[1:] - x[:-1]
        m = n - 2
        S = np.zeros(n, dtype=np.result_type(x.dtype, y.dtype))
        if m > 0 and S.dtype == np.float64:
            # the library's host restatement of the same recurrence (discoeb_natural_spline_second)
            from . import _abi
            x, y = np.ascontiguousarray(x), np.ascontiguousarray(y)
            rc = _abi.lib().discoeb_natural_spline_second(n, x.ctypes.data, y.ctypes.data, S.ctypes.data)
            if rc != 0:
                raise ValueError(f"discoeb_natural_spline_second failed with code {rc}")
        elif m > 0:  # complex-step parameters: the recurrence in numpy's complex arithmetic
            a = h[:-1]
            b = 2.0 * (h[:-1] + h[1:])
            c = h[1:]
            d = 6.0 * ((y[2:] - y[1:-1]) / h[1:] - (y[1:-1] - y[:-2]) / h[:-1])
            cp = np.zeros(m, dtype=S.dtype)
            dp = np.zeros(m, dtype=S.dtype)
            cp[0] = c[0] / b[0]
            dp[0] = d[0] / b[0]
            for i in range(1, m):
                denom = b[i] - a[i] * cp[i - 1]
                cp[i] = c[i] / denom if i < m - 1 else 0.0
                dp[i] = (d[i] - a[i] * dp[i - 1]) / denom
            Si = np.zeros(m, dtype=S.dtype)
            Si[m - 1] = dp[m - 1]
            for idx in range(m - 2, -1, -1):
                Si[idx] = dp[idx] - cp[idx] * Si[idx + 1]
            S[1:-1] = Si
        self._finish(x, y, S, integrate_from_start, uniform)

    @classmethod
    def from_table(cls, x, y, S, integrate_from_start: bool = True, uniform: bool = False):
        """The spline with knots ``x``, values ``y`` and knot second derivatives ``S`` given
        (tables computed elsewhere, e.g. by the native background)."""
        obj = cls.__new__(cls)
        x = np.asarray(x)
        y = np.asarray(y)
        S = np.asarray(S)
        obj._finish(x.astype(np.result_type(x.dtype, np.float64)), y.astype(np.result_type(y.dtype, np.float64)),
                    S.astype(np.result_type(S.dtype, np.float64)), integrate_from_start, uniform)
        return obj

    def _finish(self, x, y, S, integrate_from_start, uniform):
        n = y.shape[0]
        h = x[1:] - x[:-1]
        a_i = y[:-1]
        b_i = (y[1:] - y[:-1]) / h - h * (S[1:] + 2.0 * S[:-1]) / 6.0
        c_i = S[:-1] / 2.0
        d_i = (S[1:] - S[:-1]) / (6.0 * h)
        I_full = a_i * h + b_i * h**2 / 2 + c_i * h**3 / 3 + d_i * h**4 / 4
        self.n = n
        self.x = x
        self.y = y
        self.S = S
        self.I_cum = np.concatenate([[0.0], np.cumsum(I_full)])
        self.I_total = self.I_cum[-1]
        self.integrate_from_start = integrate_from_start
        self.uniform = uniform
        self.x0 = x[0]
        self.dx_inv = 1.0 / (x[1] - x[0])

    # -- index lookup -----------------------------------------------------------------
    def _find_index(self, x_new):
        x_new = np.real(np.asarray(x_new))
        if self.uniform:
            idx = np.floor((x_new - self.x0) * self.dx_inv).astype(np.int64)
        else:
            # number of knots strictly below x_new, minus one (== searchsorted left - 1)
            idx = np.searchsorted(self.x, x_new, side="left") - 1
        return np.minimum(np.maximum(idx, 0), self.n - 2)  # clip to [0, n-2] (np.clip's checks cost more)

    def _local(self, x_new):
        x_new = np.asarray(x_new)
        idx = self._find_index(x_new)
        x, y, S = self.x, self.y, self.S
        h = x[idx + 1] - x[idx]
        d = x_new - x[idx]
        return idx, h, d

    def evaluate(self, x_new):
        idx, h, d = self._local(x_new)
        t = d / h
        A = 1.0 - t
        B = t
        y, S = self.y, self.S
        return (A * y[idx] + B * y[idx + 1]
                + ((A**3 - A) * S[idx] + (B**3 - B) * S[idx + 1]) * (h**2) / 6.0)

    def _coeffs(self, idx, h):
        y, S = self.y, self.S
        b = (y[idx + 1] - y[idx]) / h - h * (S[idx + 1] + 2.0 * S[idx]) / 6.0
        c = S[idx] / 2.0
        dd = (S[idx + 1] - S[idx]) / (6.0 * h)
        return b, c, dd

    def derivative(self, x_new):
        idx, h, d = self._local(x_new)
        b, c, dd = self._coeffs(idx, h)
        return b + 2.0 * c * d + 3.0 * dd * d**2

    def derivative2(self, x_new):
        idx, h, d = self._local(x_new)
        b, c, dd = self._coeffs(idx, h)
        return 2.0 * c + 6.0 * dd * d

    def derivative12(self, x_new):
        idx, h, d = self._local(x_new)
        b, c, dd = self._coeffs(idx, h)
        return b + 2.0 * c * d + 3.0 * dd * d**2, 2.0 * c + 6.0 * dd * d

    def integral(self, x_new):
        idx, h, d = self._local(x_new)
        b, c, dd = self._coeffs(idx, h)
        Ip = self.y[idx] * d + b * d**2 / 2 + c * d**3 / 3 + dd * d**4 / 4
        fwd = self.I_cum[idx] + Ip
        return fwd if self.integrate_from_start else self.I_total - fwd

    # -- table export -------------------------------------------------------------------
    def table(self) -> np.ndarray:
        """``float64[3, n]`` rows (x, y, S): the layout the C ABI takes."""
        return np.stack([self.x, self.y, self.S])
