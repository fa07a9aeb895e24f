// scatt_b200.hpp -- C++ host interface over the C ABI of libscatt_b200.
//
// Mirrors the reference's per-energy pipeline for C++ callers: the result
// structs carry the field names of ScatteringResult (src/scatt/
// KMatrixExtractor.hpp:57-67), AmplitudeResult (src/scatt/
// AsymptoticAmplitudes.hpp:50-68) and DipoleResult (src/scatt/
// DipoleMatrixElement.hpp:80-91), failures throw std::runtime_error with the
// library's message as the reference's classes do (src/scatt/
// LapackInverse.hpp:73-86, AsymptoticAmplitudes.cpp:177-186), the dense
// inverse helpers keep the names of src/scatt/LapackInverse.hpp:53-178, and
// the per-step steppers those of src/scatt/GpuPropagate.hpp:83-279.
// Matrices are column-major (Eigen's default layout) in a plain vector, so
// the header needs nothing beyond the standard library and scatt_b200.h.
#pragma once

#include <array>
#include <complex>
#include <stdexcept>
#include <string>
#include <vector>

#include "scatt_b200.h"

namespace scatt_b200 {

inline void check(int rc) {
    if (rc != SCATT_OK) throw std::runtime_error(scatt_last_error());
}

// Column-major dense matrix.
struct Matrix {
    int rows = 0, cols = 0;
    std::vector<double> data;
    Matrix() = default;
    Matrix(int r, int c) : rows(r), cols(c), data((size_t)r * c, 0.0) {}
    double& operator()(int i, int j) { return data[i + (size_t)j * rows]; }
    double operator()(int i, int j) const { return data[i + (size_t)j * rows]; }
};

struct ScatteringResult {       // KMatrixExtractor::extract
    Matrix K_matrix;
    std::vector<double> eigenphases;
    double unitarity_err = 0.0;
    double K_symmetry_err = 0.0;
    bool schur_coupling_zero = false;
};

struct AmplitudeResult {        // AsymptoticAmplitudes::extract
    Matrix A, B, K;
    std::vector<double> eigenphases;
    double fit_residual_max = 0.0, fit_residual_rel = 0.0, A_minus_I_max = 0.0;
    double K_symmetry_err = 0.0, S_unitarity_err = 0.0;
    int n_fit_start = -1, n_fit_end = -1;
};

struct DipoleResult {           // DipoleMatrixElement::compute_six, one slot
    std::vector<std::complex<double>> D_reduced, D_reduced_raw;
    std::vector<double> d_raw;
    Matrix b_overlap;           // (N_psi, n_occ)
    std::vector<double> d_correction;
    double partial_sigma = 0.0;
};

struct EnergyResult {
    double E = 0.0;
    int status = SCATT_OK;
    int n_transition = 0, shifts_A = 0, shifts_S = 0, n_closed_l = 0;
    ScatteringResult kme;
    AmplitudeResult aa;
    std::array<DipoleResult, 6> dipoles;   // (L,x) (L,y) (L,z) (V,x) (V,y) (V,z)
};

// Energy-independent inputs (the preprocessing file's content); the arrays
// are C order as documented for scatt_scan_desc.
struct ScanInputs {
    int Nr = 0;
    double dr = 0.0;
    int l_cont = 0, n_occ = 0, n_orb = 0, Nlm_store = 0, Nr_store = 0;
    std::vector<double> psi_lm;     // [n_orb][Nlm_store][Nr_store]
    int init_state = -1;
    int n_H = 0;
    std::vector<double> V_H;        // [n_H][Nr]
    std::vector<double> atoms;      // [n_atoms][4]: Z, x, y, z
    double alpha_pol = 0.0, r_c = 1.5;
    int pol_form = 0;
    int n_transition = 0;
    double chi_cutoff = 1e-15;
};

// One scan on one device: static inputs uploaded once, energies solved in
// batches (replaces the stage chain of run_one_energy per energy).
class ScanSolver {
public:
    ScanSolver(const ScanInputs& in, int device = 0) : in_(in) {
        check(scatt_ctx_create(device, &ctx_));
        scatt_scan_desc d{};
        d.Nr = in.Nr;
        d.dr = in.dr;
        d.l_cont_max = in.l_cont;
        d.n_occ = in.n_occ;
        d.n_orb = in.n_orb;
        d.Nlm_store = in.Nlm_store;
        d.Nr_store = in.Nr_store;
        d.psi_lm = in_.psi_lm.data();
        d.init_state = in.init_state;
        d.n_H = in.n_H;
        d.V_H = in_.V_H.data();
        d.n_atoms = (int)(in.atoms.size() / 4);
        d.atoms = in_.atoms.data();
        d.alpha_pol = in.alpha_pol;
        d.pol_form = in.pol_form;
        d.r_c = in.r_c;
        d.n_transition = in.n_transition;
        d.chi_cutoff = in.chi_cutoff;
        try {
            check(scatt_upload_static(ctx_, &d));
            int info[5];
            check(scatt_scan_info(ctx_, info));
            n_transition_ = info[0];
            Np_ = info[1];
        } catch (...) {
            scatt_ctx_destroy(ctx_);
            throw;
        }
    }
    ~ScanSolver() {
        if (ctx_) scatt_ctx_destroy(ctx_);
    }
    ScanSolver(const ScanSolver&) = delete;
    ScanSolver& operator=(const ScanSolver&) = delete;

    int n_transition() const { return n_transition_; }
    int n_channels() const { return Np_; }

    // Solves every energy; throws on the first failing energy unless
    // raise_on_error is false (then each result carries its status).
    std::vector<EnergyResult> solve(const std::vector<double>& E, bool allow_closed_channels = false,
                                    bool raise_on_error = true) {
        scatt_solve_opts o;
        scatt_default_opts(&o);
        o.allow_closed_channels = allow_closed_channels ? 1 : 0;
        o.diagnostics = 1;
        return solve(E, o, raise_on_error);
    }

    std::vector<EnergyResult> solve(const std::vector<double>& E, const scatt_solve_opts& o,
                                    bool raise_on_error = true) {
        const int nE = (int)E.size(), Np = Np_, no = in_.n_occ;
        const size_t n2 = (size_t)Np * Np;
        std::vector<double> K(nE * n2), A(nE * n2), B(nE * n2), Kaa(nE * n2), bov((size_t)nE * Np * no),
            Dre((size_t)nE * 6 * Np), Dim((size_t)nE * 6 * Np), Rre((size_t)nE * 6 * Np), Rim((size_t)nE * 6 * Np),
            draw((size_t)nE * 6 * Np), dcor((size_t)nE * 6 * no), sig((size_t)nE * 6), ek((size_t)nE * Np),
            ea((size_t)nE * Np), diag((size_t)nE * SCATT_NDIAG);
        std::vector<int> st(nE);
        scatt_outputs out{K.data(),    A.data(),    B.data(),    Kaa.data(), bov.data(),  Dre.data(),
                          Dim.data(),  Rre.data(),  Rim.data(),  draw.data(), dcor.data(), sig.data(),
                          ek.data(),   ea.data(),   diag.data(), st.data()};
        const int rc = scatt_solve_batch(ctx_, nE, E.data(), nullptr, &o, &out);
        if (rc != SCATT_OK && raise_on_error) check(rc);
        std::vector<EnergyResult> res(nE);
        for (int e = 0; e < nE; ++e) {
            EnergyResult& r = res[e];
            const double* g = diag.data() + (size_t)e * SCATT_NDIAG;
            r.E = E[e];
            r.status = st[e];
            r.n_transition = (int)g[SCATT_DIAG_N_TRANSITION];
            r.shifts_A = (int)g[SCATT_DIAG_SHIFTS_A];
            r.shifts_S = (int)g[SCATT_DIAG_SHIFTS_S];
            r.n_closed_l = (int)g[SCATT_DIAG_N_CLOSED_L];
            r.kme.K_matrix = block(K.data() + e * n2, Np, Np);
            r.kme.eigenphases.assign(ek.begin() + (size_t)e * Np, ek.begin() + (size_t)(e + 1) * Np);
            r.kme.K_symmetry_err = g[SCATT_DIAG_K_SYMMETRY_ERR_KME];
            r.kme.unitarity_err = g[SCATT_DIAG_UNITARITY_ERR_KME];
            r.kme.schur_coupling_zero = g[SCATT_DIAG_SCHUR_COUPLING_0] != 0.0;
            r.aa.A = block(A.data() + e * n2, Np, Np);
            r.aa.B = block(B.data() + e * n2, Np, Np);
            r.aa.K = block(Kaa.data() + e * n2, Np, Np);
            r.aa.eigenphases.assign(ea.begin() + (size_t)e * Np, ea.begin() + (size_t)(e + 1) * Np);
            r.aa.fit_residual_max = g[SCATT_DIAG_FIT_RESIDUAL_MAX];
            r.aa.fit_residual_rel = g[SCATT_DIAG_FIT_RESIDUAL_REL];
            r.aa.A_minus_I_max = g[SCATT_DIAG_A_MINUS_I_MAX];
            r.aa.K_symmetry_err = g[SCATT_DIAG_K_SYMMETRY_ERR_AA];
            r.aa.S_unitarity_err = g[SCATT_DIAG_S_UNITARITY_ERR_AA];
            r.aa.n_fit_start = (int)g[SCATT_DIAG_N_FIT_START];
            r.aa.n_fit_end = (int)g[SCATT_DIAG_N_FIT_END];
            for (int s = 0; s < 6; ++s) {
                DipoleResult& d = r.dipoles[s];
                const size_t v0 = ((size_t)e * 6 + s) * Np;
                d.D_reduced.resize(Np);
                d.D_reduced_raw.resize(Np);
                d.d_raw.assign(draw.begin() + v0, draw.begin() + v0 + Np);
                for (int m = 0; m < Np; ++m) {
                    d.D_reduced[m] = {Dre[v0 + m], Dim[v0 + m]};
                    d.D_reduced_raw[m] = {Rre[v0 + m], Rim[v0 + m]};
                }
                d.b_overlap = block(bov.data() + (size_t)e * Np * no, Np, no);
                d.d_correction.assign(dcor.begin() + ((size_t)e * 6 + s) * no,
                                      dcor.begin() + ((size_t)e * 6 + s + 1) * no);
                d.partial_sigma = sig[(size_t)e * 6 + s];
            }
        }
        return res;
    }

private:
    static Matrix block(const double* p, int r, int c) {
        Matrix m(r, c);
        for (size_t i = 0; i < m.data.size(); ++i) m.data[i] = p[i];
        return m;
    }
    ScanInputs in_;
    scatt_ctx* ctx_ = nullptr;
    int n_transition_ = 0, Np_ = 0;
};

// The reference's per-radial-step seam (src/scatt/GpuPropagate.hpp:83-279):
// carried state stays on the device, one step's operands are host matrices.
class GpuForwardStepper {
public:
    GpuForwardStepper(int n_total, int device = 0) : n_(n_total) {
        check(scatt_fwd_stepper_create(device, n_total, &h_));
    }
    ~GpuForwardStepper() { scatt_fwd_stepper_destroy(h_); }
    GpuForwardStepper(const GpuForwardStepper&) = delete;
    GpuForwardStepper& operator=(const GpuForwardStepper&) = delete;
    void init_R_prev_inv(const Matrix& R) { check(scatt_fwd_stepper_init(h_, R.data.data())); }
    // Rinv_out = sym((12 W_inv - 10 I - R_prev_inv)^-1); returns max |Rinv - Rinv^T|
    double step(const Matrix& W_inv, Matrix& Rinv_out) {
        Rinv_out = Matrix(n_, n_);
        double asym = 0.0;
        check(scatt_fwd_stepper_step(h_, W_inv.data.data(), Rinv_out.data.data(), &asym));
        return asym;
    }

private:
    int n_;
    scatt_fwd_stepper* h_ = nullptr;
};

class GpuSinvStepper {
public:
    GpuSinvStepper(int n_psi, int n_f, int device = 0) : np_(n_psi) {
        check(scatt_sinv_stepper_create(device, n_psi, n_f, &h_));
    }
    ~GpuSinvStepper() { scatt_sinv_stepper_destroy(h_); }
    GpuSinvStepper(const GpuSinvStepper&) = delete;
    GpuSinvStepper& operator=(const GpuSinvStepper&) = delete;
    // Sinv = sym((A - B diag(Dinv) B^T)^-1)
    double step(const Matrix& A, const Matrix& B, const std::vector<double>& Dinv, Matrix& Sinv_out) {
        Sinv_out = Matrix(np_, np_);
        double asym = 0.0;
        check(scatt_sinv_stepper_step(h_, A.data.data(), B.data.data(), Dinv.data(), Sinv_out.data.data(), &asym));
        return asym;
    }
    // Sinv = sym(A^-1) (no exchange coupling)
    double step_inverse_only(const Matrix& A, Matrix& Sinv_out) {
        Sinv_out = Matrix(np_, np_);
        double asym = 0.0;
        check(scatt_sinv_stepper_step(h_, A.data.data(), nullptr, nullptr, Sinv_out.data.data(), &asym));
        return asym;
    }

private:
    int np_;
    scatt_sinv_stepper* h_ = nullptr;
};

class GpuBackStepper {
public:
    GpuBackStepper(int n_total, int n_psi, int device = 0) : nt_(n_total), np_(n_psi) {
        check(scatt_back_stepper_create(device, n_total, n_psi, &h_));
    }
    ~GpuBackStepper() { scatt_back_stepper_destroy(h_); }
    GpuBackStepper(const GpuBackStepper&) = delete;
    GpuBackStepper& operator=(const GpuBackStepper&) = delete;
    void init_Z(const Matrix& Z) { check(scatt_back_stepper_init(h_, Z.data.data())); }
    // Z <- Rinv Z; Y = W_inv Z; psi_out = Y[0:n_psi, :]; f_out = Y[n_psi:, :] when compute_f
    void step(const Matrix& Rinv, const Matrix& W_inv, Matrix& psi_out, Matrix* f_out, bool compute_f) {
        psi_out = Matrix(np_, np_);
        double* f = nullptr;
        if (compute_f && f_out) {
            *f_out = Matrix(nt_ - np_, np_);
            f = f_out->data.data();
        }
        check(scatt_back_stepper_step(h_, Rinv.data.data(), W_inv.data.data(), psi_out.data.data(), f));
    }
    void get_Z(Matrix& Z_out) const {
        Z_out = Matrix(nt_, np_);
        check(scatt_back_stepper_get_z(h_, Z_out.data.data()));
    }

private:
    int nt_, np_;
    scatt_back_stepper* h_ = nullptr;
};

// Dense inverses on the device, named as in LapackInverse.hpp:53-178; a
// singular or non-finite pivot throws std::runtime_error.
inline Matrix inverse_general(const Matrix& A) {
    if (A.rows != A.cols) throw std::runtime_error("inverse_general: matrix is not square");
    Matrix out(A.rows, A.cols);
    check(scatt_inverse_batched(A.rows, 1, A.data.data(), out.data.data(), 0, nullptr));
    return out;
}

inline Matrix inverse_symmetric_indefinite(const Matrix& A) {
    if (A.rows != A.cols) throw std::runtime_error("inverse_symmetric_indefinite: matrix is not square");
    Matrix out(A.rows, A.cols);
    check(scatt_inverse_batched(A.rows, 1, A.data.data(), out.data.data(), 1, nullptr));
    return out;
}

}  // namespace scatt_b200
