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

#include <algorithm>
#include <array>
#include <chrono>
#include <complex>
#include <cstddef>
#include <cstdint>
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

    // psi(n) for n_lo <= n < n_hi of every energy, by the back-propagation of
    // BackPropagator::run / get_psi (src/scatt/BackPropagator.cpp:199-802)
    // through scatt_psi_sweep: psi[e][n - n_lo] is Np x Np (rows = channel,
    // columns = solution).  The energies' other results are not kept here
    // (solve() returns them).  Throws on a failing energy.
    std::vector<std::vector<Matrix>> psi(const std::vector<double>& E, int n_lo, int n_hi, int segment = 64,
                                         bool allow_closed_channels = false) {
        std::vector<double> buf;
        psi_into(E, n_lo, n_hi, segment, allow_closed_channels, buf);
        const size_t n2 = (size_t)Np_ * Np_;
        std::vector<std::vector<Matrix>> out(E.size());
        for (size_t e = 0; e < E.size(); ++e)
            for (int n = n_lo; n < n_hi; ++n)
                out[e].push_back(block(buf.data() + (e * (size_t)(n_hi - n_lo) + (size_t)(n - n_lo)) * n2, Np_, Np_));
        return out;
    }
    // The same into one flat buffer in the C ABI's layout: energy-major, then
    // point, each Np x Np column-major.  Page-locked memory (cudaHostAlloc or
    // cudaHostRegister on out.data()) lets the copies overlap the sweep.
    void psi_into(const std::vector<double>& E, int n_lo, int n_hi, int segment, bool allow_closed_channels,
                  std::vector<double>& out) {
        scatt_solve_opts o;
        scatt_default_opts(&o);
        o.allow_closed_channels = allow_closed_channels ? 1 : 0;
        std::vector<int> st(E.size());
        scatt_outputs res{};
        res.status = st.data();
        out.assign(E.size() * (size_t)std::max(0, n_hi - n_lo) * Np_ * Np_, 0.0);
        check(scatt_psi_sweep(ctx_, &o, (int)E.size(), E.data(), nullptr, segment, n_lo, n_hi, &res, out.data()));
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

// cc_raw of one final state kappa against one intermediate state nu
// (cc_dipole::compute_cc_dipole, postprocessing/two_photon_delay/cc_dipole/
// include/CCDipole.hpp; CCDipole.cpp:294-334), length gauge, on the device
// through scatt_cc_dipole: psi_kappa[i], psi_nu[i] are psi at radial index
// ir0 + i (as ScanSolver::psi returns them, all N_psi x N_psi), pol one of
// 'x', 'y', 'z'.  Simpson weights over the whole window, r = (ir0 + i + 1) dr.
inline Matrix compute_cc_dipole(const std::vector<Matrix>& psi_kappa, const std::vector<Matrix>& psi_nu, int ir0,
                                double dr, char pol) {
    if (psi_kappa.empty() || psi_kappa.size() != psi_nu.size())
        throw std::runtime_error("compute_cc_dipole: psi_kappa and psi_nu need the same non-empty window");
    const int n = psi_kappa[0].rows;
    const size_t n2 = (size_t)n * n;
    std::vector<double> k(psi_kappa.size() * n2), v(psi_nu.size() * n2);
    for (size_t i = 0; i < psi_kappa.size(); ++i) {
        if (psi_kappa[i].rows != n || psi_kappa[i].cols != n || psi_nu[i].rows != n || psi_nu[i].cols != n)
            throw std::runtime_error("compute_cc_dipole: every psi must be N_psi x N_psi");
        std::copy(psi_kappa[i].data.begin(), psi_kappa[i].data.end(), k.begin() + i * n2);
        std::copy(psi_nu[i].data.begin(), psi_nu[i].data.end(), v.begin() + i * n2);
    }
    const int q = pol == 'x' ? 1 : pol == 'y' ? -1 : pol == 'z' ? 0 : 2;
    Matrix cc(n, n);
    check(scatt_cc_dipole(n, n, (int)psi_kappa.size(), ir0, dr, q, k.data(), 1, v.data(), cc.data.data()));
    return cc;
}

// ------------------------------------------------------------ per-step seam
// The reference's device seam -- GpuContext and the Sinv, forward and back
// steppers of src/scatt/GpuPropagate.hpp:52-279, and GpuDipoleEngine of
// src/scatt/GpuDipoleEngine.hpp:85-149 -- with their constructors, methods
// and Stats fields, over the per-step entry points of the C ABI.  The
// reference's stage classes (SchurInverter, ForwardRPropagator,
// BackPropagator, DipoleMatrixElement with use_gpu) build these objects
// exactly as written there; host/seam/scatt/ holds the two headers that put
// them into namespace scatt in place of the reference's own.
// Matrix arguments are Eigen::MatrixXd / Eigen::VectorXd or any column-major
// contiguous type with rows(), cols(), data() and resize(r, c) (size() and
// data() for vectors), or scatt_b200::Matrix / std::vector<double>.
// The carried state (R_prev^-1, Z) stays on the device between steps.
// One step is one library call on the device's stream (upload, device work,
// download); its host time is reported in the step's main timing field
// (t_inverse_ns, t_gemm_z_ns, t_gemm_ns) and the other fields stay 0.
namespace detail {
template <class M> inline int rows_of(const M& m) { return static_cast<int>(m.rows()); }
template <class M> inline int cols_of(const M& m) { return static_cast<int>(m.cols()); }
template <class M> inline const double* data_of(const M& m) { return m.data(); }
template <class M> inline double* resized(M& m, int r, int c) { m.resize(r, c); return m.data(); }
inline int rows_of(const Matrix& m) { return m.rows; }
inline int cols_of(const Matrix& m) { return m.cols; }
inline const double* data_of(const Matrix& m) { return m.data.data(); }
inline double* resized(Matrix& m, int r, int c) { m = Matrix(r, c); return m.data.data(); }
template <class V> inline int size_of(const V& v) { return static_cast<int>(v.size()); }
template <class M> inline void need_shape(const M& m, int r, int c, const char* what) {
    if (rows_of(m) != r || cols_of(m) != c)
        throw std::runtime_error(std::string(what) + ": expected a " + std::to_string(r) + " x " +
                                 std::to_string(c) + " matrix");
}
using Clock = std::chrono::steady_clock;
inline std::uint64_t ns_since(Clock::time_point t0) {
    return static_cast<std::uint64_t>(
        std::chrono::duration_cast<std::chrono::nanoseconds>(Clock::now() - t0).count());
}
}  // namespace detail

// GpuPropagate.hpp:52-80.  prefer_gpu = true throws when no CUDA device is
// visible.  prefer_gpu = false constructs without one; the reference then
// runs its host fallback, and this library has none, so a stepper built
// on such a context throws (SCATT_ERR_NO_DEVICE).
class GpuContext {
public:
    struct Info {
        std::string device_name;
        std::string platform_name;
        bool is_gpu = false;
        std::size_t global_mem_bytes = 0;     // not reported by the library: 0
    };
    explicit GpuContext(bool prefer_gpu = true, int device = 0) : device_(device) {
        int n = 0;
        if (scatt_device_count(&n) != SCATT_OK) n = 0;
        info_.platform_name = "CUDA (libscatt_b200)";
        if (device >= 0 && device < n) {
            info_.is_gpu = true;
            info_.device_name = "CUDA device " + std::to_string(device);
        } else if (prefer_gpu) {
            throw std::runtime_error("GpuContext: no CUDA device " + std::to_string(device) +
                                     " is visible (the library has no CPU fallback)");
        }
    }
    GpuContext(const GpuContext&) = delete;
    GpuContext& operator=(const GpuContext&) = delete;
    const Info& info() const { return info_; }
    void* raw_queue() const { return nullptr; }   // the library owns its streams
    int device() const { return device_; }
    static bool gpu_available() {
        int n = 0;
        return scatt_device_count(&n) == SCATT_OK && n > 0;
    }

private:
    Info info_{};
    int device_ = 0;
};

// GpuPropagate.hpp:83-150:  Rinv_n = sym((12 W_n^-1 - 10 I - Rinv_{n-1})^-1).
class GpuForwardStepper {
public:
    struct Stats {
        std::uint64_t t_upload_ns = 0, t_u_combine_ns = 0, t_inverse_ns = 0, t_download_ns = 0;
        std::uint64_t n_steps = 0;
    };
    GpuForwardStepper(GpuContext& ctx, int N_total) : ctx_(ctx), N_(N_total) {
        check(scatt_fwd_stepper_create(ctx.device(), N_total, &h_));
    }
    ~GpuForwardStepper() { scatt_fwd_stepper_destroy(h_); }
    GpuForwardStepper(const GpuForwardStepper&) = delete;
    GpuForwardStepper& operator=(const GpuForwardStepper&) = delete;

    template <class M> void init_R_prev_inv(const M& R) {
        detail::need_shape(R, N_, N_, "GpuForwardStepper::init_R_prev_inv");
        check(scatt_fwd_stepper_init(h_, detail::data_of(R)));
    }
    // Returns max |Rinv - Rinv^T| (0: the result is symmetrised exactly).
    template <class M1, class M2> double step(const M1& W_inv, M2& Rinv_out) {
        detail::need_shape(W_inv, N_, N_, "GpuForwardStepper::step");
        const auto t0 = detail::Clock::now();
        double* out = detail::resized(Rinv_out, N_, N_);
        double asym = 0.0;
        check(scatt_fwd_stepper_step(h_, detail::data_of(W_inv), out, &asym));
        stats_.t_inverse_ns += detail::ns_since(t0);
        ++stats_.n_steps;
        return asym;
    }
    // The request for an LDL^T inverse is recorded and not taken: the
    // library has one inverse (Gauss-Jordan with partial pivoting, then
    // symmetrised), whose result is bit-symmetric already.
    void enable_symmetric_inverse(bool enable) { requested_ = enable; }
    bool is_symmetric_inverse_active() const { return false; }
    bool symmetric_inverse_supported() const { return false; }
    int N_total() const { return N_; }
    const Stats& stats() const { return stats_; }
    void reset_stats() { stats_ = Stats{}; }

private:
    [[maybe_unused]] GpuContext& ctx_;
    int N_;
    bool requested_ = false;
    scatt_fwd_stepper* h_ = nullptr;
    Stats stats_{};
};

// GpuPropagate.hpp:153-227:  Sinv = sym((A - B diag(Dinv) B^T)^-1).
class GpuSinvStepper {
public:
    struct Stats {
        std::uint64_t t_upload_ns = 0, t_schur_ns = 0, t_inverse_ns = 0, t_download_ns = 0;
        std::uint64_t n_steps = 0;
    };
    GpuSinvStepper(GpuContext& ctx, int N_psi, int N_f) : ctx_(ctx), N_psi_(N_psi), N_f_(N_f) {
        check(scatt_sinv_stepper_create(ctx.device(), N_psi, N_f, &h_));
    }
    ~GpuSinvStepper() { scatt_sinv_stepper_destroy(h_); }
    GpuSinvStepper(const GpuSinvStepper&) = delete;
    GpuSinvStepper& operator=(const GpuSinvStepper&) = delete;

    template <class MA, class MB, class VD, class MO>
    double step(const MA& A, const MB& B, const VD& Dinv, MO& Sinv_out) {
        detail::need_shape(A, N_psi_, N_psi_, "GpuSinvStepper::step (A)");
        detail::need_shape(B, N_psi_, N_f_, "GpuSinvStepper::step (B)");
        if (detail::size_of(Dinv) != N_f_) throw std::runtime_error("GpuSinvStepper::step: Dinv must have N_f entries");
        return run(detail::data_of(A), detail::data_of(B), Dinv.data(), Sinv_out);
    }
    // n >= n_transition: Sinv = sym(A^-1)
    template <class MA, class MO> double step_inverse_only(const MA& A, MO& Sinv_out) {
        detail::need_shape(A, N_psi_, N_psi_, "GpuSinvStepper::step_inverse_only");
        return run(detail::data_of(A), nullptr, nullptr, Sinv_out);
    }
    int N_psi() const { return N_psi_; }
    int N_f() const { return N_f_; }
    const Stats& stats() const { return stats_; }
    void reset_stats() { stats_ = Stats{}; }

private:
    template <class MO> double run(const double* A, const double* B, const double* Dinv, MO& Sinv_out) {
        const auto t0 = detail::Clock::now();
        double* out = detail::resized(Sinv_out, N_psi_, N_psi_);
        double asym = 0.0;
        check(scatt_sinv_stepper_step(h_, A, B, Dinv, out, &asym));
        stats_.t_inverse_ns += detail::ns_since(t0);
        ++stats_.n_steps;
        return asym;
    }
    [[maybe_unused]] GpuContext& ctx_;
    int N_psi_, N_f_;
    scatt_sinv_stepper* h_ = nullptr;
    Stats stats_{};
};

// GpuPropagate.hpp:230-279:  Z <- Rinv Z;  Y = W_inv Z;  psi = Y[0:N_psi], f = Y[N_psi:].
class GpuBackStepper {
public:
    struct Stats {
        std::uint64_t t_upload_ns = 0, t_gemm_z_ns = 0, t_gemm_y_ns = 0, t_extract_ns = 0;
        std::uint64_t n_steps = 0;
    };
    GpuBackStepper(GpuContext& ctx, int N_total, int N_psi, int N_f)
        : ctx_(ctx), N_total_(N_total), N_psi_(N_psi), N_f_(N_f) {
        if (N_total != N_psi + N_f) throw std::runtime_error("GpuBackStepper: N_total must be N_psi + N_f");
        check(scatt_back_stepper_create(ctx.device(), N_total, N_psi, &h_));
    }
    ~GpuBackStepper() { scatt_back_stepper_destroy(h_); }
    GpuBackStepper(const GpuBackStepper&) = delete;
    GpuBackStepper& operator=(const GpuBackStepper&) = delete;

    template <class M> void init_Z(const M& Z) {
        detail::need_shape(Z, N_total_, N_psi_, "GpuBackStepper::init_Z");
        check(scatt_back_stepper_init(h_, detail::data_of(Z)));
    }
    template <class MR, class MW, class MP, class MF>
    void step(const MR& Rinv, const MW& W_inv, MP& psi_out, MF* f_out, bool compute_f) {
        double* f = nullptr;
        if (compute_f && f_out) f = detail::resized(*f_out, N_f_, N_psi_);
        run(Rinv, W_inv, psi_out, f);
    }
    template <class MR, class MW, class MP>
    void step(const MR& Rinv, const MW& W_inv, MP& psi_out, std::nullptr_t, bool) {
        run(Rinv, W_inv, psi_out, nullptr);
    }
    template <class M> void get_Z(M& Z_out) const {
        check(scatt_back_stepper_get_z(h_, detail::resized(Z_out, N_total_, N_psi_)));
    }
    int N_total() const { return N_total_; }
    int N_psi() const { return N_psi_; }
    int N_f() const { return N_f_; }
    const Stats& stats() const { return stats_; }
    void reset_stats() { stats_ = Stats{}; }

private:
    template <class MR, class MW, class MP> void run(const MR& Rinv, const MW& W_inv, MP& psi_out, double* f) {
        detail::need_shape(Rinv, N_total_, N_total_, "GpuBackStepper::step (Rinv)");
        detail::need_shape(W_inv, N_total_, N_total_, "GpuBackStepper::step (W_inv)");
        const auto t0 = detail::Clock::now();
        double* psi = detail::resized(psi_out, N_psi_, N_psi_);
        check(scatt_back_stepper_step(h_, detail::data_of(Rinv), detail::data_of(W_inv), psi, f));
        stats_.t_gemm_z_ns += detail::ns_since(t0);
        ++stats_.n_steps;
    }
    [[maybe_unused]] GpuContext& ctx_;
    int N_total_, N_psi_, N_f_;
    scatt_back_stepper* h_ = nullptr;
    Stats stats_{};
};

// GpuDipoleEngine.hpp:85-149:  result (n_slots x N_psi) = V (n_slots x N_psi) . psi_ir
// (N_psi x N_psi), one device GEMM per radial point (scatt_dgemm: on the
// calling thread's current CUDA device, with device buffers allocated per
// call; the batched solver computes the same contraction without this seam).
class GpuDipoleEngine {
public:
    struct Stats {
        std::uint64_t t_upload_ns = 0, t_gemm_ns = 0, t_download_ns = 0;
        std::uint64_t n_steps = 0;
    };
    GpuDipoleEngine(GpuContext& ctx, int N_psi, int n_slots) : ctx_(ctx), N_psi_(N_psi), n_slots_(n_slots) {
        if (N_psi <= 0 || n_slots <= 0) throw std::runtime_error("GpuDipoleEngine: bad sizes");
        if (ctx.device() < 0 || !GpuContext::gpu_available())
            throw std::runtime_error("GpuDipoleEngine: no CUDA device visible (the library has no CPU fallback)");
    }
    GpuDipoleEngine(const GpuDipoleEngine&) = delete;
    GpuDipoleEngine& operator=(const GpuDipoleEngine&) = delete;

    template <class MV, class MP, class MO> void step(const MV& V, const MP& psi_ir, MO& result_out) {
        detail::need_shape(V, n_slots_, N_psi_, "GpuDipoleEngine::step (V)");
        detail::need_shape(psi_ir, N_psi_, N_psi_, "GpuDipoleEngine::step (psi_ir)");
        const auto t0 = detail::Clock::now();
        double* out = detail::resized(result_out, n_slots_, N_psi_);
        check(scatt_dgemm(0, 0, n_slots_, N_psi_, N_psi_, 1.0, detail::data_of(V), n_slots_,
                          detail::data_of(psi_ir), N_psi_, 0.0, out, n_slots_));
        stats_.t_gemm_ns += detail::ns_since(t0);
        ++stats_.n_steps;
    }
    int N_psi() const { return N_psi_; }
    int n_slots() const { return n_slots_; }
    const Stats& stats() const { return stats_; }
    void reset_stats() { stats_ = Stats{}; }

private:
    [[maybe_unused]] GpuContext& ctx_;
    int N_psi_, n_slots_;
    Stats stats_{};
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
