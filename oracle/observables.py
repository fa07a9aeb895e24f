"""Test-only restatement of the reference's photoionisation observables
(postprocessing/cross_section_delay.py:195-275 and the asymmetry parameter
:350-430, constants :120-122), written
with explicit loops so it shares no code with the package's vectorised
version.  The k-derivative is numpy.gradient's second-order scheme on an
uneven grid (first order at the two ends), which the reference calls.
"""
import cmath
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


def dphi_rms(D_L, D_V):
    """cross_section_delay.py:270-275, one energy at a time."""
    out = []
    for e in range(len(D_L)):
        sw = swp = 0.0
        for a, b in zip(D_L[e], D_V[e]):
            w = abs(a) * abs(b)
            d = cmath.phase(b * a.conjugate())
            sw += w
            swp += w * d * d
        out.append(math.sqrt(swp / sw) if sw > 1e-30 else 0.0)
    return out


def beta(D_x, D_y, D_z, n_theta=40, n_phi=80):
    """cross_section_delay.py:350-430: beta = N_1 / sigma_tot - 1 on the
    Gauss-Legendre x trapezoid grid, point by point, with the real
    harmonics of oracle.angular (Gaunt.hpp:171-181); channel i is lm index i."""
    import numpy as np
    from .angular import idx_to_lm, real_Ylm
    x, w = np.polynomial.legendre.leggauss(n_theta)
    dphi = 2.0 * math.pi / n_phi
    n_ch = len(D_x[0])
    lms = [idx_to_lm(i) for i in range(n_ch)]
    out = []
    for e in range(len(D_x)):
        sig = n1 = 0.0
        for it in range(n_theta):
            th = math.acos(x[it])
            for ip in range(n_phi):
                ph = ip * dphi
                Y = [real_Ylm(l, m, th, ph) for l, m in lms]
                maps = [sum(D[e][i] * Y[i] for i in range(n_ch)) for D in (D_x, D_y, D_z)]
                kx, ky, kz = math.sin(th) * math.cos(ph), math.sin(th) * math.sin(ph), math.cos(th)
                wt = w[it] * dphi
                sig += wt * sum(abs(mp) ** 2 for mp in maps) / 3.0
                n1 += wt * abs(maps[0] * kx + maps[1] * ky + maps[2] * kz) ** 2
        out.append(n1 / sig - 1.0 if sig > 1e-30 else 0.0)
    return out
