// host_tables_shim.cpp -- extern "C" access to the library's host-side table
// builders (spion-emol_b200/csrc/tables.cpp) for the CPU tests.  The tests
// compile this file together with tables.cpp and angular.cpp, with the flags
// the library uses, and compare each table with the oracle.  CSR builders
// return their entry count and fill the arrays only when it fits in `cap`.
#include <cstring>

#include "tables.hpp"

using namespace scatt;

extern "C" {

void t_vsigma(int Nr, double dr, int l_max, int n_H, const double* V_H, int n_atoms,
              const double* atoms, double* out) {
    const std::vector<double> T = build_vsigma(Nr, dr, l_max, n_H, V_H, n_atoms, atoms);
    std::memcpy(out, T.data(), T.size() * sizeof(double));
}

int t_gaunt_pairs(int l_max, int cap, int* row, int* col, int* ptr, int* sig, double* G) {
    const PairCSR P = build_gaunt_pairs(l_max);
    const int nnz = (int)P.G.size();
    if (nnz > cap) return nnz;
    std::memcpy(row, P.row.data(), P.row.size() * sizeof(int));
    std::memcpy(col, P.col.data(), P.col.size() * sizeof(int));
    std::memcpy(ptr, P.ptr.data(), P.ptr.size() * sizeof(int));
    std::memcpy(sig, P.sig.data(), nnz * sizeof(int));
    std::memcpy(G, P.G.data(), nnz * sizeof(double));
    return nnz;
}

int t_exchange(int n_mu, int n_sigma, int n_lambda, int cap, int* ptr, int* lam, double* G,
               int* n_lambda_max) {
    const ExchCSR X = build_exchange(n_mu, n_sigma, n_lambda);
    const int nnz = (int)X.G.size();
    if (nnz > cap) return nnz;
    std::memcpy(ptr, X.ptr.data(), X.ptr.size() * sizeof(int));
    std::memcpy(lam, X.lam.data(), nnz * sizeof(int));
    std::memcpy(G, X.G.data(), nnz * sizeof(double));
    *n_lambda_max = X.n_lambda_max;
    return nnz;
}

int t_dipole(int n_mu, int n_lambda, int qi, int cap, int* ptr, int* nu, double* a, double* c) {
    const DipCSR D = build_dipole_tables(n_mu, n_lambda);
    const int nnz = (int)D.a[qi].size();
    if (nnz > cap) return nnz;
    std::memcpy(ptr, D.ptr[qi].data(), D.ptr[qi].size() * sizeof(int));
    std::memcpy(nu, D.nu[qi].data(), nnz * sizeof(int));
    std::memcpy(a, D.a[qi].data(), nnz * sizeof(double));
    std::memcpy(c, D.c[qi].data(), nnz * sizeof(double));
    return nnz;
}

void t_simpson(int n, double h, double* w) {
    const std::vector<double> v = simpson_weights(n, h);
    std::memcpy(w, v.data(), v.size() * sizeof(double));
}

void t_five_point(const double* f, int n, double dr, double* df) { five_point_derivative(f, n, dr, df); }

}  // extern "C"
