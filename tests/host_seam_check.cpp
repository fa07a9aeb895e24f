// host_seam_check.cpp -- the reference's stage classes' calls into the
// device seam (SchurInverter.cpp:191-313, ForwardRPropagator.cpp:261-312,
// BackPropagator.cpp:559-645, DipoleMatrixElement.cpp:742-827), written as
// there, compiled against spion-emol_b200/host/seam instead of the
// reference's GpuPropagate.hpp / GpuDipoleEngine.hpp.  Eigen is not in this
// image, so a minimal stand-in with Eigen's column-major MatrixXd / VectorXd
// surface is defined first.  Without a GPU the program checks the no-device
// behaviour: GpuContext(true) throws, GpuContext(false) constructs, and the
// first stepper built on it throws the library's message.  Exit 0 = pass.
#include <cstddef>
#include <iostream>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace Eigen {
using Index = std::ptrdiff_t;
class MatrixXd {
public:
    MatrixXd() = default;
    MatrixXd(Index r, Index c) { resize(r, c); }
    void resize(Index r, Index c) { r_ = r; c_ = c; v_.assign(static_cast<std::size_t>(r * c), 0.0); }
    Index rows() const { return r_; }
    Index cols() const { return c_; }
    double* data() { return v_.data(); }
    const double* data() const { return v_.data(); }
    double& operator()(Index i, Index j) { return v_[static_cast<std::size_t>(i + j * r_)]; }

private:
    Index r_ = 0, c_ = 0;
    std::vector<double> v_;
};
class VectorXd {
public:
    explicit VectorXd(Index n = 0) : v_(static_cast<std::size_t>(n), 0.0) {}
    Index size() const { return static_cast<Index>(v_.size()); }
    double* data() { return v_.data(); }
    const double* data() const { return v_.data(); }
    double& operator()(Index i) { return v_[static_cast<std::size_t>(i)]; }

private:
    std::vector<double> v_;
};
}  // namespace Eigen

#include "scatt/GpuDipoleEngine.hpp"
#include "scatt/GpuPropagate.hpp"

namespace scatt {

// One use of every seam call, in the reference's own forms.
void stage_calls(bool has_f_) {
    const int N_psi = 2, N_f = 2, N_tot = N_psi + N_f, n_slots = 3;
    std::unique_ptr<GpuContext> gpu_ctx = std::make_unique<GpuContext>(/*prefer_gpu=*/false);
    std::cout << gpu_ctx->info().device_name << " " << (gpu_ctx->info().global_mem_bytes >> 30) << "\n";

    // SchurInverter
    struct WS {
        Eigen::MatrixXd A, B, Sinv;
        Eigen::VectorXd Dinv;
    } w;
    w.A.resize(N_psi, N_psi);
    w.B.resize(N_psi, N_f);
    w.Dinv = Eigen::VectorXd(N_f);
    std::unique_ptr<GpuSinvStepper> sinv = std::make_unique<GpuSinvStepper>(*gpu_ctx, N_psi, N_f);
    sinv->step(w.A, w.B, w.Dinv, w.Sinv);
    sinv->step_inverse_only(w.A, w.Sinv);

    // ForwardRPropagator
    Eigen::MatrixXd Rinv_prev(N_tot, N_tot), W_inv_host(N_tot, N_tot), Rinv_n;
    std::unique_ptr<GpuForwardStepper> fwd = std::make_unique<GpuForwardStepper>(*gpu_ctx, N_tot);
    fwd->init_R_prev_inv(Rinv_prev);
    fwd->enable_symmetric_inverse(true);
    const bool active = fwd->is_symmetric_inverse_active();
    const double asym = fwd->step(W_inv_host, Rinv_n);
    std::cout << active << asym << fwd->stats().t_inverse_ns << fwd->N_total() << "\n";

    // BackPropagator
    Eigen::MatrixXd Z(N_tot, N_psi), psi_gpu, f_gpu;
    std::unique_ptr<GpuBackStepper> back = std::make_unique<GpuBackStepper>(*gpu_ctx, N_tot, N_psi, N_f);
    back->init_Z(Z);
    back->step(Rinv_n, W_inv_host, psi_gpu, has_f_ ? &f_gpu : nullptr, has_f_);
    back->step(Rinv_n, W_inv_host, psi_gpu, nullptr, false);
    back->get_Z(Z);

    // DipoleMatrixElement
    Eigen::MatrixXd V_gpu(n_slots, N_psi), psi_ir(N_psi, N_psi), R_gpu;
    std::unique_ptr<GpuDipoleEngine> gpu_eng = std::make_unique<GpuDipoleEngine>(*gpu_ctx, N_psi, n_slots);
    gpu_eng->step(V_gpu, psi_ir, R_gpu);
    std::cout << gpu_eng->stats().n_steps << "\n";
}

}  // namespace scatt

int main() {
    if (scatt::GpuContext::gpu_available()) {
        std::cout << "compiled; a device is visible, the no-device checks do not apply\n";
        return 0;
    }
    try {
        scatt::GpuContext ctx(/*prefer_gpu=*/true);
        std::cerr << "GpuContext(true) constructed without a device\n";
        return 10;
    } catch (const std::runtime_error& e) {
        if (std::string(e.what()).find("no CUDA device") == std::string::npos) return 11;
    }
    try {
        scatt::stage_calls(true);
        std::cerr << "a stepper was built without a device\n";
        return 12;
    } catch (const std::runtime_error& e) {
        if (std::string(e.what()).find("no CUDA device") == std::string::npos) {
            std::cerr << e.what() << "\n";
            return 13;
        }
    }
    std::cout << "ok\n";
    return 0;
}
