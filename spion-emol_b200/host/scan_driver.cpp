// scan_driver -- command-line use of the C++ host interface (scatt_b200.hpp).
//
//   scan_driver solve   <inputs.bin> <results.bin>
//   scan_driver inverse <matrix.bin> <inverse.bin>
//   scan_driver stepper <n>      a GpuForwardStepper step and a GpuDipoleEngine product with known answers
//
// inputs.bin (little endian): 13 int32
//   Nr l_cont n_occ n_orb Nlm_store Nr_store init_state n_H n_atoms pol_form
//   n_transition n_energy allow_closed_channels
// then float64: dr alpha_pol r_c chi_cutoff, psi_lm [n_orb][Nlm_store][Nr_store],
// V_H [n_H][Nr], atoms [n_atoms][4], energies [n_energy].
// results.bin: int32 Np, then per energy float64: status, K (Np x Np,
// column-major), A, B, then for the six dipole slots Re D, Im D (Np each),
// then the six partial sigmas.
// matrix.bin: int32 n, float64 A (n x n column-major); inverse.bin: the inverse.
// Failures print the library's message to stderr and exit with status 2.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <vector>

#include "scatt_b200.hpp"

namespace {

template <class T>
void read_n(std::ifstream& f, T* p, size_t n) {
    f.read(reinterpret_cast<char*>(p), (std::streamsize)(n * sizeof(T)));
    if (!f) throw std::runtime_error("scan_driver: truncated input file");
}

template <class T>
void write_n(std::ofstream& f, const T* p, size_t n) {
    f.write(reinterpret_cast<const char*>(p), (std::streamsize)(n * sizeof(T)));
}

int run_solve(const char* in_path, const char* out_path) {
    std::ifstream f(in_path, std::ios::binary);
    if (!f) throw std::runtime_error(std::string("scan_driver: cannot open ") + in_path);
    int h[13];
    read_n(f, h, 13);
    scatt_b200::ScanInputs in;
    in.Nr = h[0];
    in.l_cont = h[1];
    in.n_occ = h[2];
    in.n_orb = h[3];
    in.Nlm_store = h[4];
    in.Nr_store = h[5];
    in.init_state = h[6];
    in.n_H = h[7];
    const int n_atoms = h[8];
    in.pol_form = h[9];
    in.n_transition = h[10];
    const int nE = h[11];
    const bool allow_closed = h[12] != 0;
    double d[4];
    read_n(f, d, 4);
    in.dr = d[0];
    in.alpha_pol = d[1];
    in.r_c = d[2];
    in.chi_cutoff = d[3];
    in.psi_lm.resize((size_t)in.n_orb * in.Nlm_store * in.Nr_store);
    read_n(f, in.psi_lm.data(), in.psi_lm.size());
    in.V_H.resize((size_t)in.n_H * in.Nr);
    read_n(f, in.V_H.data(), in.V_H.size());
    in.atoms.resize((size_t)n_atoms * 4);
    read_n(f, in.atoms.data(), in.atoms.size());
    std::vector<double> E(nE);
    read_n(f, E.data(), E.size());

    scatt_b200::ScanSolver solver(in, 0);
    const std::vector<scatt_b200::EnergyResult> res = solver.solve(E, allow_closed);
    std::ofstream o(out_path, std::ios::binary);
    const int Np = solver.n_channels();
    write_n(o, &Np, 1);
    for (const auto& r : res) {
        const double status = r.status;
        write_n(o, &status, 1);
        write_n(o, r.kme.K_matrix.data.data(), r.kme.K_matrix.data.size());
        write_n(o, r.aa.A.data.data(), r.aa.A.data.size());
        write_n(o, r.aa.B.data.data(), r.aa.B.data.size());
        for (const auto& dp : r.dipoles) {
            std::vector<double> re(Np), im(Np);
            for (int m = 0; m < Np; ++m) {
                re[m] = dp.D_reduced[m].real();
                im[m] = dp.D_reduced[m].imag();
            }
            write_n(o, re.data(), re.size());
            write_n(o, im.data(), im.size());
        }
        for (const auto& dp : r.dipoles) write_n(o, &dp.partial_sigma, 1);
    }
    return 0;
}

int run_inverse(const char* in_path, const char* out_path) {
    std::ifstream f(in_path, std::ios::binary);
    if (!f) throw std::runtime_error(std::string("scan_driver: cannot open ") + in_path);
    int n = 0;
    read_n(f, &n, 1);
    scatt_b200::Matrix A(n, n);
    read_n(f, A.data.data(), A.data.size());
    const scatt_b200::Matrix X = scatt_b200::inverse_general(A);
    std::ofstream o(out_path, std::ios::binary);
    write_n(o, X.data.data(), X.data.size());
    return 0;
}

}  // namespace

// The per-step seam on exact cases, built as the reference's stage classes
// build it: a forward step of order n from W_inv = I / 2 and R_prev_inv = 0
// gives Rinv = (6 I - 10 I)^-1 = -I / 4, and the dipole engine's product
// V . (2 I) = 2 V of small integers.  Prints the largest error of each.
int run_stepper(int n) {
    scatt_b200::GpuContext ctx(true);
    scatt_b200::GpuForwardStepper f(ctx, n);
    scatt_b200::Matrix W(n, n), R;
    for (int i = 0; i < n; ++i) W(i, i) = 0.5;
    f.step(W, R);
    double err = 0.0;
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) err = std::max(err, std::abs(R(i, j) - (i == j ? -0.25 : 0.0)));
    const int slots = 3;
    scatt_b200::GpuDipoleEngine eng(ctx, n, slots);
    scatt_b200::Matrix V(slots, n), psi(n, n), out;
    for (int j = 0; j < n; ++j) {
        psi(j, j) = 2.0;
        for (int s = 0; s < slots; ++s) V(s, j) = s + j;
    }
    eng.step(V, psi, out);
    double err_d = 0.0;
    for (int j = 0; j < n; ++j)
        for (int s = 0; s < slots; ++s) err_d = std::max(err_d, std::abs(out(s, j) - 2.0 * (s + j)));
    std::cout << err << " " << err_d << "\n";
    return (err < 1e-15 && err_d == 0.0 && f.stats().n_steps == 1 && eng.stats().n_steps == 1) ? 0 : 3;
}

int main(int argc, char** argv) {
    if (argc == 3 && std::strcmp(argv[1], "stepper") == 0) {
        try {
            return run_stepper(std::atoi(argv[2]));
        } catch (const std::exception& ex) {
            std::cerr << ex.what() << "\n";
            return 2;
        }
    }
    if (argc != 4 || (std::strcmp(argv[1], "solve") != 0 && std::strcmp(argv[1], "inverse") != 0)) {
        std::cerr << "usage: scan_driver solve|inverse <input> <output> | stepper <n>\n";
        return 1;
    }
    try {
        return std::strcmp(argv[1], "solve") == 0 ? run_solve(argv[2], argv[3]) : run_inverse(argv[2], argv[3]);
    } catch (const std::exception& ex) {
        std::cerr << ex.what() << "\n";
        return 2;
    }
}
