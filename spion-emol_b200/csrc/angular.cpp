// angular.cpp -- angular algebra for the host-side table precompute.
//
// Replaces src/angular/Gaunt.hpp (gaunt_real over GSL's
// gsl_sf_coupling_3j) and the dipole helpers of
// src/scatt/DipoleMatrixElement.cpp:80-95.
//
// Wigner 3j.  Racah's formula written with binomial coefficients,
//   (j1 j2 j3; m1 m2 m3) = (-1)^(j1-j2-m3)
//       * sqrt( prod (j_i + m_i)! (j_i - m_i)! / ((J+1)! a! (b+d)! (c+e)!) )
//       * sum_k (-1)^k C(a, k) C(b+d, b-k) C(c+e, c-k),
// a = j1+j2-j3, b = j1-m1, c = j2+m2, d = j3-j2+m1, e = j3-j1-m2, J = j1+j2+j3.
// The alternating integer sum is evaluated in long double; when its
// cancellation could cost accuracy it is redone exactly with a small
// arbitrary-precision integer, so every value is accurate to ~1 ulp.
// Results are memoised (thread-safe) because the table builders ask for the
// same symbols many times.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "angular.hpp"

namespace scatt {

namespace {

// ---------------------------------------------------------- tiny bignum
struct Big {
    std::vector<uint32_t> d;   // little endian magnitude
    bool neg = false;
    static Big from(uint64_t v) {
        Big b;
        while (v) { b.d.push_back(uint32_t(v)); v >>= 32; }
        return b;
    }
    bool zero() const { return d.empty(); }
    void trim() { while (!d.empty() && d.back() == 0) d.pop_back(); }
};

void mul_small(Big& a, uint32_t m) {
    uint64_t carry = 0;
    for (auto& x : a.d) {
        const uint64_t v = uint64_t(x) * m + carry;
        x = uint32_t(v);
        carry = v >> 32;
    }
    if (carry) a.d.push_back(uint32_t(carry));
}

void div_small(Big& a, uint32_t m) {   // exact division
    uint64_t rem = 0;
    for (size_t i = a.d.size(); i-- > 0;) {
        const uint64_t cur = (rem << 32) | a.d[i];
        a.d[i] = uint32_t(cur / m);
        rem = cur % m;
    }
    a.trim();
}

Big mul(const Big& a, const Big& b) {
    Big r;
    if (a.zero() || b.zero()) return r;
    r.d.assign(a.d.size() + b.d.size(), 0);
    for (size_t i = 0; i < a.d.size(); ++i) {
        uint64_t carry = 0;
        for (size_t j = 0; j < b.d.size(); ++j) {
            const uint64_t v = uint64_t(a.d[i]) * b.d[j] + r.d[i + j] + carry;
            r.d[i + j] = uint32_t(v);
            carry = v >> 32;
        }
        size_t k = i + b.d.size();
        while (carry) {
            const uint64_t v = uint64_t(r.d[k]) + carry;
            r.d[k] = uint32_t(v);
            carry = v >> 32;
            ++k;
        }
    }
    r.trim();
    return r;
}

int cmp_mag(const Big& a, const Big& b) {
    if (a.d.size() != b.d.size()) return a.d.size() < b.d.size() ? -1 : 1;
    for (size_t i = a.d.size(); i-- > 0;)
        if (a.d[i] != b.d[i]) return a.d[i] < b.d[i] ? -1 : 1;
    return 0;
}

Big add_mag(const Big& a, const Big& b) {
    Big r;
    const size_t n = std::max(a.d.size(), b.d.size());
    r.d.resize(n + 1);
    uint64_t carry = 0;
    for (size_t i = 0; i < n; ++i) {
        const uint64_t v = uint64_t(i < a.d.size() ? a.d[i] : 0) + (i < b.d.size() ? b.d[i] : 0) + carry;
        r.d[i] = uint32_t(v);
        carry = v >> 32;
    }
    r.d[n] = uint32_t(carry);
    r.trim();
    return r;
}

Big sub_mag(const Big& a, const Big& b) {   // |a| >= |b|
    Big r;
    r.d.resize(a.d.size());
    int64_t borrow = 0;
    for (size_t i = 0; i < a.d.size(); ++i) {
        int64_t v = int64_t(a.d[i]) - (i < b.d.size() ? int64_t(b.d[i]) : 0) - borrow;
        borrow = v < 0;
        if (v < 0) v += (int64_t(1) << 32);
        r.d[i] = uint32_t(v);
    }
    r.trim();
    return r;
}

Big add_signed(const Big& a, const Big& b) {
    if (a.neg == b.neg) { Big r = add_mag(a, b); r.neg = a.neg && !r.zero(); return r; }
    if (cmp_mag(a, b) >= 0) { Big r = sub_mag(a, b); r.neg = a.neg && !r.zero(); return r; }
    Big r = sub_mag(b, a);
    r.neg = b.neg && !r.zero();
    return r;
}

Big binom_big(int n, int k) {
    Big r = Big::from(1);
    if (k < 0 || k > n) return Big();
    k = std::min(k, n - k);
    for (int i = 1; i <= k; ++i) {
        mul_small(r, uint32_t(n - k + i));
        div_small(r, uint32_t(i));
    }
    return r;
}

long double big_to_ld(const Big& b) {
    long double v = 0.0L;
    for (size_t i = b.d.size(); i-- > 0;) v = v * 4294967296.0L + (long double)b.d[i];
    return b.neg ? -v : v;
}

long double lfact(int n) { return lgammal((long double)n + 1.0L); }

long double lbinom(int n, int k) { return lfact(n) - lfact(k) - lfact(n - k); }

double w3j_compute(int j1, int j2, int j3, int m1, int m2, int m3) {
    const int a = j1 + j2 - j3, b = j1 - m1, c = j2 + m2;
    const int d = j3 - j2 + m1, e = j3 - j1 - m2;
    const int J = j1 + j2 + j3;
    const int kmin = std::max({0, -d, -e});
    const int kmax = std::min({a, b, c});
    if (kmin > kmax) return 0.0;
    // alternating sum in long double, with a cancellation estimate
    long double s = 0.0L, tmax = 0.0L;
    for (int k = kmin; k <= kmax; ++k) {
        const long double t = expl(lbinom(a, k) + lbinom(b + d, b - k) + lbinom(c + e, c - k));
        tmax = std::max(tmax, t);
        s += (k & 1) ? -t : t;
    }
    const long double lpre = 0.5L * (lfact(j1 + m1) + lfact(j1 - m1) + lfact(j2 + m2) + lfact(j2 - m2)
                                     + lfact(j3 + m3) + lfact(j3 - m3) - lfact(J + 1) - lfact(a)
                                     - lfact(b + d) - lfact(c + e));
    const long double rel_err = (kmax - kmin + 1) * 4e-18L * tmax / (fabsl(s) + 1e-4000L);
    if (rel_err > 1e-17L || s == 0.0L) {
        Big S;
        for (int k = kmin; k <= kmax; ++k) {
            Big t = mul(mul(binom_big(a, k), binom_big(b + d, b - k)), binom_big(c + e, c - k));
            t.neg = (k & 1) && !t.zero();
            S = add_signed(S, t);
        }
        if (S.zero()) return 0.0;
        // S may exceed the long double range only far beyond l ~ 1000
        const long double ls = logl(fabsl(big_to_ld(S)));
        const long double v = expl(ls + lpre);
        const double sign = (((j1 - j2 - m3) & 1) ? -1.0 : 1.0) * (S.neg ? -1.0 : 1.0);
        return sign * (double)v;
    }
    const long double v = expl(logl(fabsl(s)) + lpre);
    const double sign = (((j1 - j2 - m3) & 1) ? -1.0 : 1.0) * (s < 0 ? -1.0 : 1.0);
    return sign * (double)v;
}

std::mutex g_mu;
std::unordered_map<uint64_t, double> g_w3j;

uint64_t key3j(int j1, int j2, int j3, int m1, int m2) {
    return (uint64_t(j1) << 50) | (uint64_t(j2) << 38) | (uint64_t(j3) << 26) |
           (uint64_t(m1 + 2048) << 13) | uint64_t(m2 + 2048);
}

}  // namespace

double wigner3j(int j1, int j2, int j3, int m1, int m2, int m3) {
    if (m1 + m2 + m3 != 0) return 0.0;
    if (j1 < 0 || j2 < 0 || j3 < 0) return 0.0;
    if (std::abs(m1) > j1 || std::abs(m2) > j2 || std::abs(m3) > j3) return 0.0;
    if (j3 < std::abs(j1 - j2) || j3 > j1 + j2) return 0.0;
    const uint64_t key = key3j(j1, j2, j3, m1, m2);
    {
        std::lock_guard<std::mutex> lk(g_mu);
        auto it = g_w3j.find(key);
        if (it != g_w3j.end()) return it->second;
    }
    const double v = w3j_compute(j1, j2, j3, m1, m2, m3);
    std::lock_guard<std::mutex> lk(g_mu);
    g_w3j.emplace(key, v);
    return v;
}

// Gaunt.hpp:65-87
double gaunt_complex_no_conj(int l1, int m1, int l2, int m2, int l3, int m3) {
    if (m1 + m2 + m3 != 0) return 0.0;
    if (std::abs(l1 - l2) > l3) return 0.0;
    if (l1 + l2 < l3) return 0.0;
    if ((l1 + l2 + l3) & 1) return 0.0;
    const double w000 = wigner3j(l1, l2, l3, 0, 0, 0);
    const double wmmm = wigner3j(l1, l2, l3, m1, m2, m3);
    if (!std::isfinite(w000) || !std::isfinite(wmmm)) return 0.0;
    const double pre = std::sqrt((2.0 * l1 + 1.0) * (2.0 * l2 + 1.0) * (2.0 * l3 + 1.0) / (4.0 * M_PI));
    return pre * w000 * wmmm;
}

namespace {
struct Cplx { double re, im; };
inline Cplx cmul(Cplx a, Cplx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline double phase(int m) { return (m & 1) ? -1.0 : 1.0; }
// Gaunt.hpp:93-110
inline Cplx U_real_to_complex(int mR, int mC) {
    const double s = M_SQRT1_2;
    if (mR == 0) return mC == 0 ? Cplx{1.0, 0.0} : Cplx{0.0, 0.0};
    if (mR > 0) {
        if (mC == -mR) return {s, 0.0};
        if (mC == mR) return {s * phase(mR), 0.0};
        return {0.0, 0.0};
    }
    const int p = -mR;
    if (mC == -p) return {0.0, s};
    if (mC == p) return {0.0, -s * phase(p)};
    return {0.0, 0.0};
}
inline bool nz(Cplx z) { return z.re != 0.0 || z.im != 0.0; }
}  // namespace

// Gaunt.hpp:114-135 -- the complex-m sum only visits the two m values each
// real harmonic is made of (+-|m|), which is exactly the set of non-zero U.
double gaunt_real(int l1, int mR1, int l2, int mR2, int l3, int mR3) {
    if (std::abs(l1 - l2) > l3 || l1 + l2 < l3) return 0.0;
    if ((l1 + l2 + l3) & 1) return 0.0;
    if (std::abs(mR1) > l1 || std::abs(mR2) > l2 || std::abs(mR3) > l3) return 0.0;
    const int a1 = std::abs(mR1), a2 = std::abs(mR2), a3 = std::abs(mR3);
    if (a3 != a1 + a2 && a3 != std::abs(a1 - a2)) return 0.0;
    double re = 0.0, im = 0.0;
    const int c1[2] = {-a1, a1}, c2[2] = {-a2, a2};
    for (int i1 = 0; i1 < (a1 ? 2 : 1); ++i1) {
        const int m1 = c1[i1];
        const Cplx U1 = U_real_to_complex(mR1, m1);
        if (!nz(U1)) continue;
        for (int i2 = 0; i2 < (a2 ? 2 : 1); ++i2) {
            const int m2 = c2[i2];
            const Cplx U2 = U_real_to_complex(mR2, m2);
            if (!nz(U2)) continue;
            const int m3 = -(m1 + m2);
            if (m3 < -l3 || m3 > l3) continue;
            const Cplx U3 = U_real_to_complex(mR3, m3);
            if (!nz(U3)) continue;
            const double Gc = gaunt_complex_no_conj(l1, m1, l2, m2, l3, m3);
            if (Gc == 0.0) continue;
            const Cplx p = cmul(cmul(U1, U2), U3);
            re += p.re * Gc;
            im += p.im * Gc;
        }
    }
    (void)im;
    return re;
}

// Gaunt.hpp:148-181
double real_Ylm(int l, int m, double theta, double phi) {
    if (l < 0 || std::abs(m) > l) return 0.0;
    const int am = std::abs(m);
    const double s = std::sin(theta), c = std::cos(theta);
    double S_mm = 1.0 / std::sqrt(4.0 * M_PI);
    for (int k = 1; k <= am; ++k) S_mm *= std::sqrt((2.0 * k + 1.0) / (2.0 * k)) * s;
    double S = S_mm;
    if (l > am) {
        double S_prev = S_mm;
        double S_cur = std::sqrt(2.0 * am + 3.0) * c * S_mm;
        if (l == am + 1) {
            S = S_cur;
        } else {
            double S_pp = S_prev;
            S_prev = S_cur;
            for (int k = am + 2; k <= l; ++k) {
                const double a = std::sqrt((4.0 * k * k - 1.0) / (double(k) * k - am * am));
                const double b = std::sqrt((double(k - 1) * (k - 1) - am * am) / (4.0 * (k - 1.0) * (k - 1.0) - 1.0));
                const double Sk = a * (c * S_prev - b * S_pp);
                S_pp = S_prev;
                S_prev = Sk;
            }
            S = S_prev;
        }
    }
    if (m == 0) return S;
    if (m > 0) return std::sqrt(2.0) * S * std::cos(m * phi);
    return std::sqrt(2.0) * S * std::sin(am * phi);
}

double angular_dipole(int l_mu, int m_mu, int q, int l_nu, int m_nu) {
    return std::sqrt(4.0 * M_PI / 3.0) * gaunt_real(l_mu, m_mu, 1, q, l_nu, m_nu);
}

double velocity_coef(int l_mu, int l_nu) {
    if (l_mu == l_nu + 1) return -double(l_nu + 1);
    if (l_mu == l_nu - 1) return double(l_nu);
    return 0.0;
}

}  // namespace scatt
