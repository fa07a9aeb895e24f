// riccati.cuh -- Riccati-Bessel x j_l(x) and Riccati-Neumann x y_l(x),
// callable on host and device.
//
// The reference uses GSL's gsl_sf_bessel_jl_e / gsl_sf_bessel_yl_e times x
// (ForwardRPropagator.cpp:64-75, KMatrixExtractor.cpp:50-73,
// AsymptoticAmplitudes.cpp:39-62), treating GSL underflow as 0.  This is an
// independent implementation of the textbook methods (Abramowitz & Stegun
// 10.1):
//   * power series  j_l(x) = x^l / (2l+1)!! * sum_k (-x^2/2)^k / (k! prod_{i<=k}(2l+2i+1))
//     for small x (prefactor evaluated in log space, so it only underflows
//     where the true value is below the double range);
//   * upward recurrence  f_{n+1} = (2n+1)/x f_n - f_{n-1}  for j_l when x > l
//     and for y_l always (stable directions);
//   * Miller's downward recurrence for j_l when x <= l, normalised by
//     j_0 = sin x / x (or j_1 when sin x is small).
#pragma once

#include <cmath>

#ifdef __CUDACC__
#define SCATT_HD __host__ __device__ __forceinline__
#else
#define SCATT_HD inline
#endif

namespace scatt {

SCATT_HD double sph_j_series(int l, double x) {
    // log((2l+1)!!) = sum_{i=1..l} log(2i+1)
    double logdf = 0.0;
    for (int i = 1; i <= l; ++i) logdf += log(2.0 * i + 1.0);
    const double lp = l * log(x) - logdf;
    if (lp < -745.0) return 0.0;
    double pre;
    if (lp > -650.0) {
        pre = 1.0;                       // x^l / (2l+1)!! as a product of l factors
        for (int i = 1; i <= l; ++i) pre *= x / (2.0 * i + 1.0);
    } else {
        pre = exp(lp);
    }
    const double y = -0.5 * x * x;
    double term = 1.0, sum = 1.0;
    for (int k = 1; k < 200; ++k) {
        term *= y / (k * (2.0 * l + 2.0 * k + 1.0));
        sum += term;
        if (fabs(term) < 1e-18 * fabs(sum)) break;
    }
    return pre * sum;
}

SCATT_HD double sph_j(int l, double x) {
    if (l < 0) return 0.0;
    if (x * x < 1.0 + 0.5 * l) return sph_j_series(l, x);
    const double s = sin(x), c = cos(x);
    const double j0 = s / x;
    if (l == 0) return j0;
    const double j1 = s / (x * x) - c / x;
    if (l == 1) return j1;
    if (x > (double)l) {
        double jm = j0, jc = j1;
        for (int n = 1; n < l; ++n) {
            const double jn = (2.0 * n + 1.0) / x * jc - jm;
            jm = jc;
            jc = jn;
        }
        return jc;
    }
    // Miller: start well above max(l, x)
    int L = l + 40 + (int)(2.0 * sqrt((double)l + x));
    double fp1 = 0.0, f = 1e-250, fl = 0.0, f0 = 0.0, f1 = 0.0;
    for (int n = L; n >= 1; --n) {
        const double fm1 = (2.0 * n + 1.0) / x * f - fp1;   // f_{n-1}
        fp1 = f;
        f = fm1;
        if (n - 1 == l) fl = f;
        if (n - 1 == 1) f1 = f;
        if (fabs(f) > 1e250) {
            f *= 1e-250; fp1 *= 1e-250; fl *= 1e-250; f1 *= 1e-250;
        }
    }
    f0 = f;
    if (l == 1) fl = f1;
    if (fabs(j0) > 0.1 * fabs(j1) || fabs(f1) == 0.0) return fl * (j0 / f0);
    return fl * (j1 / f1);
}

SCATT_HD double sph_y(int l, double x) {
    const double s = sin(x), c = cos(x);
    const double y0 = -c / x;
    if (l == 0) return y0;
    const double y1 = -c / (x * x) - s / x;
    double ym = y0, yc = y1;
    for (int n = 1; n < l; ++n) {
        const double yn = (2.0 * n + 1.0) / x * yc - ym;
        ym = yc;
        yc = yn;
    }
    return yc;
}

// x j_l(x); 0 for x < 1e-300 (ForwardRPropagator.cpp:67).
SCATT_HD double riccati_j(int l, double x) {
    if (x < 1e-300) return 0.0;
    return x * sph_j(l, x);
}

// x y_l(x); callers never pass x ~ 0 (the reference throws there).
SCATT_HD double riccati_y(int l, double x) {
    return x * sph_y(l, x);
}

}  // namespace scatt
