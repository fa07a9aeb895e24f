"""Test-only restatement of the reference's photoionisation observables
(postprocessing/cross_section_delay.py:195-263, constants :120-122), written
with explicit loops so it shares no code with the package's vectorised
version.  The k-derivative is numpy.gradient's second-order scheme on an
uneven grid (first order at the two ends), which the reference calls.
"""
import math

C_AU = 137.036


def d_dk(k, f):
    """Derivative of the samples f(k) (numpy.gradient, edge_order 1)."""
    n = len(k)
    out = [0j] * n
    out[0] = (f[1] - f[0]) / (k[1] - k[0])
    out[n - 1] = (f[n - 1] - f[n - 2]) / (k[n - 1] - k[n - 2])
    for i in range(1, n - 1):
        hm, hp = k[i] - k[i - 1], k[i + 1] - k[i]
        out[i] = (hm * hm * f[i + 1] - hp * hp * f[i - 1] + (hp * hp - hm * hm) * f[i]) / (hm * hp * (hm + hp))
    return out


def cross_section(k, D, omega, gauge):
    """cross_section_delay.py:195-221."""
    out = []
    for e in range(len(k)):
        s2 = sum(abs(x) ** 2 for x in D[e])
        if gauge == "length":
            out.append(8.0 * math.pi * omega[e] / (C_AU * k[e]) * s2)
        else:
            out.append(8.0 * math.pi / (C_AU * k[e] * omega[e]) * s2)
    return out


def time_delay(k, D):
    """cross_section_delay.py:227-263 (default sign convention)."""
    ne, nc = len(k), len(D[0])
    dE = [[0j] * nc for _ in range(ne)]
    for c in range(nc):
        col = d_dk(k, [D[e][c] for e in range(ne)])
        for e in range(ne):
            dE[e][c] = col[e] / k[e]
    out = []
    for e in range(ne):
        num = sum((D[e][c].conjugate() * dE[e][c]) for c in range(nc)).imag
        den = sum(abs(D[e][c]) ** 2 for c in range(nc))
        out.append(num / den if den > 1e-30 else 0.0)
    return out
