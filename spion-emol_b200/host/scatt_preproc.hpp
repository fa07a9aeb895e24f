// scatt_preproc.hpp -- C++ interface to the preprocessing steps of the
// library, named after the reference's preprocessing functions so that its
// driver (preprocessing/src/main_preprocess.cpp) can call them in place of
// its own:
//
//   read_molden        preproc::molden::MoldenParser::parse (molden/Molden.hpp)
//   project_samples    preproc::sce::project (sce/SCE.hpp:122-266), with the
//                      samples of F on the grid in place of the F3D callback
//   project_basis      build_basis + evaluate_mo / evaluate_density
//                      (basis/MoldenBasis.hpp) + project, and the local
//                      exchange of potential/LocalExchange.hpp
//   build_V_H          preproc::potential::build_V_H (potential/Hartree.hpp)
//
// Matrices are the Matrix of scatt_b200.hpp (column-major), shaped as the
// reference's Eigen results: F_lm and V_H as (Nlm, Nr).  Errors throw
// std::runtime_error with the library's message; without a CUDA device the
// device steps throw its no-device message (there is no CPU path).
#pragma once

#include <string>
#include <vector>

#include "scatt_b200.hpp"

namespace scatt_b200 {
namespace preproc {

struct Shell {                    // one contracted shell, raw coefficients as in the file
    double center[3];
    int l;
    std::vector<double> exponents, coeffs;
};

struct Orbitals {                 // one spin's MOs: C is n_mo x nbf, row i = MO i
    Matrix C;
    std::vector<double> occ, energy;
};

struct MoldenFile {
    std::vector<double> atoms;    // n_atoms x (Z, x, y, z), bohr
    std::vector<Shell> shells;
    int nbf = 0;
    Orbitals alpha, beta;
};

inline MoldenFile read_molden(const std::string& path) {
    scatt_molden* h = nullptr;
    check(scatt_molden_open(path.c_str(), &h));
    struct Closer {
        scatt_molden* h;
        ~Closer() { scatt_molden_close(h); }
    } closer{h};
    int info[7];
    check(scatt_molden_info(h, info));
    MoldenFile f;
    f.nbf = info[2];
    f.atoms.assign((size_t)info[0] * 4, 0.0);
    check(scatt_molden_atoms(h, f.atoms.data()));
    const int ns = info[1], np = info[5];
    std::vector<int> l(ns), npr(ns);
    std::vector<double> cen((size_t)ns * 3), ex(np > 0 ? np : 1), cf(np > 0 ? np : 1);
    check(scatt_molden_shells(h, l.data(), npr.data(), cen.data(), ex.data(), cf.data()));
    for (int i = 0, p = 0; i < ns; p += npr[i], ++i) {
        Shell s{{cen[3 * i], cen[3 * i + 1], cen[3 * i + 2]}, l[i], {}, {}};
        s.exponents.assign(ex.begin() + p, ex.begin() + p + npr[i]);
        s.coeffs.assign(cf.begin() + p, cf.begin() + p + npr[i]);
        f.shells.push_back(std::move(s));
    }
    for (int spin = 0; spin < 2; ++spin) {
        Orbitals& o = spin ? f.beta : f.alpha;
        const int n = info[3 + spin];
        if (!n) continue;
        std::vector<double> rows((size_t)n * f.nbf);
        o.occ.assign(n, 0.0);
        o.energy.assign(n, 0.0);
        check(scatt_molden_mos(h, spin, rows.data(), o.occ.data(), o.energy.data()));
        o.C = Matrix(n, f.nbf);
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < f.nbf; ++j) o.C(i, j) = rows[(size_t)i * f.nbf + j];
    }
    return f;
}

namespace detail {
// (Nlm, Nr) column-major from the library's row-major [Nlm][Nr]
inline Matrix from_rows(const double* p, int rows, int cols) {
    Matrix m(rows, cols);
    for (int i = 0; i < rows; ++i)
        for (int k = 0; k < cols; ++k) m(i, k) = p[(size_t)i * cols + k];
    return m;
}
}  // namespace detail

// F_lm (Nlm x Nr) of samples[(k n_theta + i) n_phi + j] = F(r_k, theta_i, phi_j)
// on the grid of scatt_sce_grid(Lmax).
inline Matrix project_samples(const std::vector<double>& samples, int Lmax, int Nr, int chunk = 0) {
    const int nlm = (Lmax + 1) * (Lmax + 1);
    if ((long)samples.size() != (long)Nr * (Lmax + 1) * 2 * (Lmax + 1))
        throw std::runtime_error("project_samples: samples must hold Nr x (Lmax + 1) x 2 (Lmax + 1) values");
    std::vector<double> out((size_t)nlm * Nr);
    check(scatt_sce_project(Lmax, Nr, chunk, samples.data(), out.data()));
    return detail::from_rows(out.data(), nlm, Nr);
}

struct BasisExpansion {
    std::vector<Matrix> orbitals;  // n_mo x (Nlm, Nr)
    Matrix rho;                    // (Nlm, Nr)
    Matrix V_x;                    // (Nlm, Nr); empty without local exchange
};

// vx_form: 0 none, 1 Slater, 2 Kohn-Sham.  The grid: r_k = r0 + k dr, k < Nr, around `origin`.
inline BasisExpansion project_basis(const MoldenFile& f, const Orbitals& mos, int Lmax, int Nr, double r0,
                                    double dr, const double origin[3], int vx_form = 0, int chunk = 0) {
    const int ns = (int)f.shells.size(), nlm = (Lmax + 1) * (Lmax + 1), n_mo = mos.C.rows;
    std::vector<int> l(ns), npr(ns);
    std::vector<double> cen((size_t)ns * 3), ex, cf;
    for (int i = 0; i < ns; ++i) {
        const Shell& s = f.shells[i];
        l[i] = s.l;
        npr[i] = (int)s.exponents.size();
        for (int k = 0; k < 3; ++k) cen[3 * i + k] = s.center[k];
        ex.insert(ex.end(), s.exponents.begin(), s.exponents.end());
        cf.insert(cf.end(), s.coeffs.begin(), s.coeffs.end());
    }
    std::vector<double> C((size_t)n_mo * f.nbf);
    for (int i = 0; i < n_mo; ++i)
        for (int j = 0; j < f.nbf; ++j) C[(size_t)i * f.nbf + j] = mos.C(i, j);
    std::vector<double> orb((size_t)n_mo * nlm * Nr), rho((size_t)nlm * Nr), vx(vx_form ? (size_t)nlm * Nr : 0);
    check(scatt_sce_basis(Lmax, Nr, r0, dr, origin, ns, l.data(), npr.data(), cen.data(), ex.data(), cf.data(),
                          n_mo, C.data(), mos.occ.data(), vx_form, chunk, orb.data(), rho.data(),
                          vx_form ? vx.data() : nullptr));
    BasisExpansion b;
    for (int i = 0; i < n_mo; ++i) b.orbitals.push_back(detail::from_rows(orb.data() + (size_t)i * nlm * Nr, nlm, Nr));
    b.rho = detail::from_rows(rho.data(), nlm, Nr);
    if (vx_form) b.V_x = detail::from_rows(vx.data(), nlm, Nr);
    return b;
}

// V_H (Nlm x Nr, Nlm = (Lmax + 1)^2) from rho_lm (>= Nlm rows, Nr columns) on r_k = r0 + k dr.
inline Matrix build_V_H(const Matrix& rho_lm, double dr, int Lmax, double r0 = 0.0) {
    const int nlm = (Lmax + 1) * (Lmax + 1), Nr = rho_lm.cols;
    std::vector<double> rows((size_t)rho_lm.rows * Nr), out((size_t)nlm * Nr);
    for (int i = 0; i < rho_lm.rows; ++i)
        for (int k = 0; k < Nr; ++k) rows[(size_t)i * Nr + k] = rho_lm(i, k);
    check(scatt_hartree(Lmax, rho_lm.rows, Nr, r0, dr, rows.data(), out.data()));
    return detail::from_rows(out.data(), nlm, Nr);
}

}  // namespace preproc
}  // namespace scatt_b200
