// tables.hpp -- host-side builders of the per-scan tables (see tables.cpp).
#pragma once

#include <vector>

namespace scatt {

struct PairCSR {              // V_{mu',mu} = sum_sigma G V_sigma over pairs mu >= mu'
    std::vector<int> row, col, ptr, sig;
    std::vector<double> G;
};

struct ExchCSR {              // G_combined[(mu*n_sigma + sigma), lambda]
    std::vector<int> ptr, lam;
    std::vector<double> G;
    int n_lambda_max = 0;
};

struct DipCSR {               // per q in (x, y, z): Ang(mu, nu) with velocity coefficients
    std::vector<int> ptr[3], nu[3];
    std::vector<double> a[3], c[3];
};

std::vector<double> build_vsigma(int Nr, double dr, int l_max, int n_H, const double* V_H,
                                 int n_atoms, const double* atoms);
PairCSR build_gaunt_pairs(int l_max);
ExchCSR build_exchange(int n_mu, int n_sigma, int n_lambda);
DipCSR build_dipole_tables(int n_mu, int n_lambda);
std::vector<double> simpson_weights(int n, double h);
void five_point_derivative(const double* f, int n, double dr, double* df);

}  // namespace scatt
