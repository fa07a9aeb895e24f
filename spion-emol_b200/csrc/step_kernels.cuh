// step_kernels.cuh -- per-energy device state of a batch and the kernels of
// one radial step (see solver.cu for the orchestration).
#pragma once

#include "common.cuh"

namespace scatt {

// Per-energy device state of a batch (one entry per energy).
struct EnergyDev {
    double E, c, k;        // energy, 1 + h^2 E / 6, sqrt(2E)
    int Np, Nt;            // continuum channels, Np + Nf
    int l_cont;
    int shiftsA, shiftsS;  // Johnson stability shifts applied (SchurInverter.cpp:264-272, 364-371)
    double deltaA;         // shift applied to A at the current step
    int err_code, err_step;
    const double* lmA;     // lambda_min(-h^2/6 V(n)) for n < stab_n (this Np)
    const double* lmS;     // lambda_min(-h^2/6 V(n) - Bs(n) B(n)^T)
    double *S, *Sw, *Sinv, *T, *F;
    double *Ra, *Rw, *Rinv0, *Rinv1, *G0, *G1;
    double *tailR, *tailS, *psiT;
    int *sigS, *ridS, *stS, *sigR, *ridR, *stR;
    double *PS, *PR;       // two-level panel windows (4 x Np x 64, 4 x Nt x 64: two sets for look-ahead)
    int *sgS, *sgR;        // composite row maps of the windows (4 x Np, 4 x Nt)
};

// Batch-level constants and shared per-step buffers.
struct BatchDev {
    int count;
    int Nr, N, n_tr, n_pts, n_start, n_s, stab_n;
    int Np_max, Nf, n_sigma, n_occ, Krows, n_lambda, n_lambda_ex;
    double dr, h2_6, h2_12, W_min, margin;
    double alpha_pol, r_c;
    int pol_form;
    // shared tables
    const double* vsig;     // [ir][sigma]
    int n_exp, n_pairs;
    const int *pair_row, *pair_col, *pair_ptr, *pair_sig;
    const double* pair_G;
    const int *ex_ptr, *ex_lam;
    const double* ex_G;
    const double* chi;      // [n][lambda][i]
    const double* Ctab;     // [n][K x Np_max]
    const int* l_of_mu;
    const int* l_sigma;
    // shared per-step buffers
    double *V, *vdiag1, *B, *Bs, *Dinv;
    // entry arrays written by k_prepare
    GemmEntry *gmS, *gmT, *gmF, *gmG1, *gmG2, *gmG3;
    GjEntry *gjS, *gjR;
    EnergyDev* ed;
};

}  // namespace scatt
