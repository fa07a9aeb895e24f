// scan.cuh -- device-resident state of one energy scan (static tables) and
// of one batch of energies solved together.
#pragma once

#include <memory>
#include <vector>

#include "common.cuh"
#include "devbuf.cuh"

namespace scatt {

constexpr int N_SLOTS = 6;   // (L,x) (L,y) (L,z) (V,x) (V,y) (V,z): DipoleMatrixElement.cpp:603-610

// Energy-independent tables of a scan, built once by scatt_upload_static.
struct ScanTables {
    // grid / channel set (for the largest l_cont of the scan)
    int Nr = 0;
    double dr = 0.0;
    int l_max = 0;          // largest l_cont
    int l_x = 0;            // exchange cutoff min(l_cont, 10) (shared by the scan)
    int n_sigma = 0;
    int n_occ = 0;
    int Np_max = 0;         // (l_max + 1)^2
    int n_lambda = 0;       // (l_max + l_x + 1)^2
    int Nf = 0;             // n_occ * n_sigma
    int n_tr = 0;           // n_transition
    int n_exp = 0;          // (2 l_max + 1)^2
    double alpha_pol = 0.0, r_c = 1.5;
    int pol_form = 0;
    const double* dV = nullptr;   // optional caller device array added to V(n): [Nr][Np_max][Np_max]
    // potential: V_sigma(r_ir) [ir][sigma], Gaunt pair CSR
    DevBuf<double> vsig;
    int n_pairs = 0;
    DevBuf<int> pair_row, pair_col, pair_ptr, pair_sig;
    DevBuf<double> pair_G;
    // exchange coupling CSR G_combined[(mu*n_sigma + sigma), lambda]
    int n_lambda_ex = 0;
    DevBuf<int> ex_ptr, ex_lam;
    DevBuf<double> ex_G;
    // chi[n][lambda][i] = (n dr) * F_{i,lambda}(n dr), n < n_tr
    DevBuf<double> chi;
    // dipole rows C_n (K x Np_max, ld K) for n < n_tr, K = 6 + n_occ
    int Krows = 0;
    DevBuf<double> Ctab;
    std::vector<double> d_corr;     // [alpha][slot]
    std::vector<double> spin;       // N_alpha
    std::vector<int> l_of_mu;       // l of each continuum channel
    DevBuf<int> d_l_of_mu;          // l of mu (Np_max)
    DevBuf<int> d_l_sigma;          // l of sigma (n_sigma)
    // Johnson stability: lambda_min(-h^2/6 V(n)) and lambda_min(-h^2/6 V(n) - Bs B^T)
    // for n < stab_n, per continuum size (cached per l_cont)
    struct StabEig { int l_cont; std::vector<double> lmA, lmS; };
    std::vector<StabEig> stab;
    bool ready = false;
};

struct SolveStats {
    double device_s = 0.0, rinv_s = 0.0, sweep_s = 0.0, post_s = 0.0;
    double rinv_calls = 0.0;
    double rinv_flops = 0.0;   // 2 n^3 summed over the matrices of the sampled inversions
    unsigned long long launches = 0;
};

struct Context {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::unique_ptr<ScanTables> tab;
    SolveStats stats;
};

}  // namespace scatt
