"""Riccati-Bessel functions for the oracle.

The reference evaluates j_l / y_l with GSL (gsl_sf_bessel_jl_e /
gsl_sf_bessel_yl_e) and multiplies by x:
  * ForwardRPropagator.cpp:64-75   riccati_besselJ_  (x < 1e-300 -> 0)
  * KMatrixExtractor.cpp:50-73     riccati_j_ / riccati_y_
  * AsymptoticAmplitudes.cpp:39-62 riccati_j_ / riccati_y_
GSL underflow (GSL_EUNDRFLW) is accepted by the reference and returns 0.
Here scipy.special.spherical_jn / spherical_yn stand in for GSL; the
oracle's values are pinned to mpmath in tests/test_oracle_golden.py.
"""
from __future__ import annotations

import numpy as np
from scipy.special import spherical_jn, spherical_yn


def riccati_j(l, x):
    """x * j_l(x); 0 for x < 1e-300 (ForwardRPropagator.cpp:67)."""
    x = np.asarray(x, dtype=np.float64)
    l = np.asarray(l)
    out = np.where(x < 1e-300, 0.0, x * spherical_jn(l, np.where(x < 1e-300, 1.0, x)))
    return out if out.ndim else float(out)


def riccati_y(l, x):
    """x * y_l(x); the reference throws for x < 1e-300 (KMatrixExtractor.cpp:62-65)."""
    x = np.asarray(x, dtype=np.float64)
    if np.any(x < 1e-300):
        raise ValueError("riccati_y called at x ~ 0")
    out = x * spherical_yn(np.asarray(l), x)
    return out if np.ndim(out) else float(out)
