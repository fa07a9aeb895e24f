// step_kernels.cuh -- per-energy device state of a batch and the kernels of
// one radial step (see solver.cu for the orchestration).
#pragma once

#include "common.cuh"

namespace scatt {

// Radial steps whose Schur complements are formed and inverted together
// (they depend on V(n), B(n) and E only, not on the R-ratio recurrence).
constexpr int SCHUR_CHUNK = 8;

// Per-energy device state of a batch (one entry per energy).
struct EnergyDev {
    double E, c, k;        // energy, 1 + h^2 E / 6, sqrt(2E)
    int Np, Nt;            // continuum channels, Np + Nf
    int l_cont;
    int shiftsA, shiftsS;  // Johnson stability shifts applied (SchurInverter.cpp:264-272, 364-371)
    double deltaA;         // scratch after the sweep (Schur coupling flag)
    double deltaAc[SCHUR_CHUNK];  // shift applied to A at each step of the current chunk
    int err_code, err_step;
    const double* lmA;     // lambda_min(-h^2/6 V(n)) for n < stab_n (this Np)
    const double* lmS;     // lambda_min(-h^2/6 V(n) - Bs(n) B(n)^T)
    double *S, *Sw, *Sinv;  // SCHUR_CHUNK slots of Np x Np each (one per step of the chunk)
    double *T, *F;
    double *Ra, *Rw, *Rinv0, *Rinv1, *G0, *G1;
    double *tailR, *tailS, *psiT;
    int *sigS, *ridS, *stS;   // SCHUR_CHUNK slots (Np, Np, 4 ints each)
    int *sigR, *ridR, *stR;
    double *PS, *PR;       // two-level panel windows (4 x Np x 64 per Schur slot, 4 x Nt x 64)
    int *sgS, *sgR;        // composite row maps of the windows (4 x Np per Schur slot, 4 x Nt)
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
    // shared per-step buffers: the current step's slot of the chunk arrays
    double *V, *vdiag1, *B, *Bs, *Dinv;
    // chunk arrays (SCHUR_CHUNK slots of V, B, Bs, D^-1) and the chunk's first step
    double *Vc, *Bc, *Bsc, *Dinvc;
    int cn0;
    // entry arrays written by k_prepare
    GemmEntry *gmS, *gmT, *gmF, *gmG1, *gmG2, *gmG3;
    GjEntry *gjS, *gjR;
    EnergyDev* ed;
};

}  // namespace scatt
