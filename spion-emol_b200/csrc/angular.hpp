// angular.hpp -- host-side angular algebra (see angular.cpp).
#pragma once

#include <cmath>

namespace scatt {

// idx = l^2 + l + m (src/angular/Gaunt.hpp:46-52)
inline int lm_to_idx(int l, int m) { return l * l + l + m; }
inline void idx_to_lm(int idx, int& l, int& m) {
    l = static_cast<int>(std::sqrt(static_cast<double>(idx)));
    if ((l + 1) * (l + 1) <= idx) ++l;
    m = idx - l * l - l;
}
inline int l_of(int idx) { int l, m; idx_to_lm(idx, l, m); return l; }

double wigner3j(int j1, int j2, int j3, int m1, int m2, int m3);
double gaunt_complex_no_conj(int l1, int m1, int l2, int m2, int l3, int m3);
double gaunt_real(int l1, int m1, int l2, int m2, int l3, int m3);
double real_Ylm(int l, int m, double theta, double phi);
double angular_dipole(int l_mu, int m_mu, int q, int l_nu, int m_nu);
double velocity_coef(int l_mu, int l_nu);

}  // namespace scatt
