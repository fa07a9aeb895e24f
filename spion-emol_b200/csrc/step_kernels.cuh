// step_kernels.cuh -- per-energy device state of a scan's slots and the
// kernels of one radial step (see solver.cu for the orchestration).
//
// The energies in flight sit in slots; slots form phase groups.  Every
// energy of a group is at the same radial step, and different groups may be
// at different steps, so a scan can keep its slots full while energies
// finish and new ones enter (one group after another) instead of waiting for
// the slowest batch.
#pragma once

#include "common.cuh"

namespace scatt {

// Radial steps whose Schur complements are formed and inverted together
// (they depend on V(n), B(n) and E only, not on the R-ratio recurrence).
constexpr int SCHUR_CHUNK = 8;

// Most phase groups a scan may have.
constexpr int MAX_GROUPS = 64;

// Device state of one phase group: the radial step at the start of its
// current chunk and its share of the per-step V, B, Bs, D^-1 slots.  Only
// kernels change n0 once a chunk is running (k_advance), so a chunk's
// launches read their step from device memory and take no per-step
// arguments.
struct GroupDev {
    int n0;          // first radial step of the current chunk; < 0: no chunk
    int C;           // steps in the current chunk (<= SCHUR_CHUNK)
    double *Vc, *Bc, *Bsc, *Dinvc;   // SCHUR_CHUNK slots each (ld Np_max)
    double* vdiag1;  // diagonal of V(n + 1) for the analytic start
};

// Per-energy device state of a batch (one entry per energy).
struct EnergyDev {
    double E, c, k;        // energy, 1 + h^2 E / 6, sqrt(2E)
    int Np, Nt;            // continuum channels, Np + Nf
    int l_cont;
    int shiftsA, shiftsS;  // Johnson stability shifts applied (SchurInverter.cpp:264-272, 364-371)
    double deltaA;         // scratch after the sweep (Schur coupling flag)
    double deltaAc[SCHUR_CHUNK];  // shift applied to A at each step of the current chunk
    int err_code, err_step;
    int grp;               // phase group of this slot
    int live;              // 1 while the slot holds an energy
    // segment mode (the adjoint's recomputation of steps [seg_lo, seg_hi)):
    // Rinv(n), Sinv(n) and H(n)^T = G(n-1)^T + C_n E_psi^T W^-1(n) of those
    // steps go to segR / segS / segH (segH[n - seg_lo]); seg_lo == seg_hi: off
    double *segR, *segS, *segH;
    int seg_lo, seg_hi;
    double* stabd;         // when set: the shift applied to A and to S at each n < stab_n
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
    // forward accumulation of the amplitude fit (no window store: tailR == nullptr):
    // GA0 / GA1 (2 Np x N_t, ld 2 Np) hold G_A(n-1)^T by parity, with
    // G_A(n)^T = (G_A(n-1)^T + D_AB(n) E_psi W^-1(n)) Rinv(n) over the window, so that
    // [A; B] = G_A(N-1)^T Z_N; wAB [i][2][Np] are the fit weights of window point
    // n_s + i; Mab [l][8] the 2 x 2 normal-matrix inverse, closed flag, det, max
    double *GA0, *GA1, *wAB, *Mab;
};

// Scan-level constants, static tables and the slot / group arrays.
struct BatchDev {
    int count;              // slots
    int ngroups;
    int n_stop;             // chunks end before this step (N + 1 for a whole sweep)
    int Nr, N, n_tr, n_pts, n_start, n_s, stab_n;
    int ne_fit, nfit;       // fit window [n_s, ne_fit] and its length
    int Np_max, Nf, n_sigma, n_occ, Krows, n_lambda, n_lambda_ex;
    double dr, h2_6, h2_12, W_min, margin;
    double alpha_pol, r_c;
    int pol_form;
    const double* dV;       // optional additive V(n) perturbation (upper triangle read)
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
    GroupDev* grp;          // ngroups entries
    // entry arrays written by k_prepare
    GemmEntry *gmS, *gmT, *gmF, *gmG1, *gmG2, *gmG3, *gmGA;
    GjEntry *gjS, *gjR;
    EnergyDev* ed;
};

}  // namespace scatt
