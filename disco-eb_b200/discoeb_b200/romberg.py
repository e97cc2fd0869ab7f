"""Romberg quadrature with 2**divmax panels, the rule the reference takes from
``jax_cosmo.scipy.integrate.romb`` (used at ``background.py:183-186`` and
``thermodynamics_recfast.py:488``).

Published method: trapezoid sums on 1, 2, 4, ... 2**divmax panels combined by
Richardson extrapolation R[i][k] = (4**k R[i][k-1] - R[i-1][k-1]) / (4**k - 1);
the result is R[divmax][divmax].
"""
from __future__ import annotations

import numpy as np


def romb(f, a, b, divmax: int = 6):
    rng = b - a
    ordsum = 0.5 * (f(np.asarray(a, dtype=np.float64)) + f(np.asarray(b, dtype=np.float64)))
    prev = [rng * ordsum]
    n = 1
    for i in range(1, divmax + 1):
        n *= 2
        ntosum = n // 2
        h = rng / ntosum
        pts = a + 0.5 * h + h * np.arange(ntosum)
        ordsum = ordsum + np.sum(f(pts))
        row = [rng * ordsum / n]
        for k in range(1, i + 1):
            p = 4.0 ** k
            row.append((p * row[k - 1] - prev[k - 1]) / (p - 1.0))
        prev = row
    return prev[-1]
