// steppers.cu -- the reference's per-radial-step device seam, kept as a
// compatibility layer over this library's kernels (src/scatt/GpuPropagate.hpp:
// GpuForwardStepper, GpuSinvStepper, GpuBackStepper).  Each stepper keeps
// its carried state on the device (R_prev^-1, Z) and exchanges one step's
// operands with host buffers, column-major FP64, as the reference's do.
// The batched solver (scatt_solve_batch) does not use these: they serve
// callers and checks written against the per-step interface.
#include <cmath>
#include <string>
#include <vector>

#include "common.cuh"
#include "devbuf.cuh"

using namespace scatt;

namespace scatt {
namespace {

// U = 12 W - 10 I - Rprev  (the matrix the forward step inverts)
__global__ void k_fwd_assemble(const double* __restrict__ W, const double* __restrict__ Rprev,
                               double* __restrict__ U, int n) {
    const size_t total = (size_t)n * n;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total;
         idx += (size_t)gridDim.x * blockDim.x) {
        const size_t i = idx % n, j = idx / n;
        U[idx] = 12.0 * W[idx] - (i == j ? 10.0 : 0.0) - Rprev[idx];
    }
}

// Bs[:, f] = B[:, f] * Dinv[f]
__global__ void k_scale_cols(const double* __restrict__ B, const double* __restrict__ Dinv,
                             double* __restrict__ Bs, int rows, int cols) {
    const size_t total = (size_t)rows * cols;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total;
         idx += (size_t)gridDim.x * blockDim.x)
        Bs[idx] = B[idx] * Dinv[idx / rows];
}

// One-matrix inverse with its own workspace (look-ahead sized).
struct Inverter {
    int n = 0;
    DevBuf<double> A, W, P;
    DevBuf<int> sig, rid, st, sgt;
    DevBuf<GjEntry> ent;
    int setup(int order, double* out) {
        n = order;
        const size_t nn = (size_t)n * n;
        SCATT_TRY(A.alloc(nn));
        SCATT_TRY(W.alloc(nn));
        SCATT_TRY(P.alloc((size_t)4 * n * GJ_WINDOW_MAX));
        SCATT_TRY(sig.alloc(n));
        SCATT_TRY(rid.alloc(n));
        SCATT_TRY(st.alloc(2));
        SCATT_TRY(sgt.alloc((size_t)4 * n));
        const std::vector<GjEntry> e{GjEntry{A.p, W.p, out, sig.p, rid.p, st.p, n, n, n, P.p, sgt.p}};
        SCATT_TRY(ent.upload(e));
        // the upload ran on the legacy stream; the steppers work on their own
        SCATT_CUDA_TRY(cudaDeviceSynchronize());
        return SCATT_OK;
    }
    // inverts A (destroyed) into out; status words copied to the host
    int run(bool symmetrize, cudaStream_t s, const char* who) {
        SCATT_CUDA_TRY(cudaMemsetAsync(st.p, 0, 2 * sizeof(int), s));
        SCATT_TRY(gj_inverse_selected(ent.p, 1, n, symmetrize, s, true));
        int h[2] = {0, 0};
        SCATT_CUDA_TRY(cudaMemcpyAsync(h, st.p, sizeof(h), cudaMemcpyDeviceToHost, s));
        SCATT_CUDA_TRY(cudaStreamSynchronize(s));
        if (h[0] == DEV_SINGULAR) {
            set_last_error(std::string(who) + ": singular pivot at column " + std::to_string(h[1]));
            return SCATT_ERR_SINGULAR;
        }
        if (h[0] == DEV_NONFINITE) {
            set_last_error(std::string(who) + ": non-finite pivot at column " + std::to_string(h[1]));
            return SCATT_ERR_NONFINITE;
        }
        return SCATT_OK;
    }
};

int grid_for(size_t total) { return (int)std::min<size_t>((total + 255) / 256, 148 * 8); }

double max_asym(const double* M, int n) {
    double m = 0.0;
    for (int j = 0; j < n; ++j)
        for (int i = j + 1; i < n; ++i) m = std::fmax(m, std::fabs(M[i + (size_t)j * n] - M[j + (size_t)i * n]));
    return m;
}

}  // namespace
}  // namespace scatt

struct scatt_fwd_stepper {
    int device = 0, n = 0;
    cudaStream_t s = nullptr;
    DevBuf<double> W, Rprev, Rout;
    Inverter inv;
};

struct scatt_sinv_stepper {
    int device = 0, np = 0, nf = 0;
    cudaStream_t s = nullptr;
    DevBuf<double> B, Bs, Dinv, Sout;
    DevBuf<GemmEntry> gm;
    Inverter inv;
};

struct scatt_back_stepper {
    int device = 0, nt = 0, np = 0, nf = 0;
    cudaStream_t s = nullptr;
    DevBuf<double> R, W, Z0, Z1, Y;
    DevBuf<GemmEntry> gm;
    bool z_ready = false;
};

namespace {

template <class T>
int open_stepper(int device, T* h) {
    SCATT_TRY(require_device());
    SCATT_CUDA_TRY(cudaSetDevice(device));
    h->device = device;
    SCATT_CUDA_TRY(cudaStreamCreateWithFlags(&h->s, cudaStreamNonBlocking));
    return SCATT_OK;
}

template <class T>
void close_stepper(T* h) {
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->s) cudaStreamSynchronize(h->s);
    if (h->s) cudaStreamDestroy(h->s);
    delete h;
}

int gemm_one(DevBuf<GemmEntry>& slot, const GemmEntry& e, int opA, int opB, cudaStream_t s) {
    SCATT_CUDA_TRY(cudaMemcpyAsync(slot.p, &e, sizeof(GemmEntry), cudaMemcpyHostToDevice, s));
    SCATT_TRY(gemm_batched(slot.p, 1, e.M, e.N, opA, opB, s));
    return SCATT_OK;
}

}  // namespace

extern "C" {

// ------------------------------------------------------------- forward
int scatt_fwd_stepper_create(int device, int n_total, scatt_fwd_stepper** out) {
    if (!out || n_total <= 0) {
        set_last_error("scatt_fwd_stepper_create: bad arguments");
        return SCATT_ERR_ARG;
    }
    *out = nullptr;
    auto* h = new scatt_fwd_stepper();
    int st = open_stepper(device, h);
    const size_t nn = (size_t)n_total * n_total;
    h->n = n_total;
    if (st == SCATT_OK) st = h->W.alloc(nn);
    if (st == SCATT_OK) st = h->Rprev.alloc(nn);
    if (st == SCATT_OK) st = h->Rout.alloc(nn);
    if (st == SCATT_OK) st = h->inv.setup(n_total, h->Rout.p);
    if (st == SCATT_OK) st = SCATT_CUDA_TRY_RET(cudaMemsetAsync(h->Rprev.p, 0, nn * sizeof(double), h->s));
    if (st != SCATT_OK) {
        close_stepper(h);
        return st;
    }
    *out = h;
    return SCATT_OK;
}

int scatt_fwd_stepper_destroy(scatt_fwd_stepper* h) {
    close_stepper(h);
    return SCATT_OK;
}

int scatt_fwd_stepper_init(scatt_fwd_stepper* h, const double* rprev_inv) {
    if (!h || !rprev_inv) return SCATT_ERR_ARG;
    SCATT_CUDA_TRY(cudaSetDevice(h->device));
    SCATT_CUDA_TRY(cudaMemcpyAsync(h->Rprev.p, rprev_inv, (size_t)h->n * h->n * sizeof(double),
                                   cudaMemcpyHostToDevice, h->s));
    SCATT_CUDA_TRY(cudaStreamSynchronize(h->s));
    return SCATT_OK;
}

int scatt_fwd_stepper_step(scatt_fwd_stepper* h, const double* w_inv, double* rinv_out, double* max_asym_out) {
    if (!h || !w_inv || !rinv_out) return SCATT_ERR_ARG;
    SCATT_CUDA_TRY(cudaSetDevice(h->device));
    const size_t nn = (size_t)h->n * h->n;
    SCATT_CUDA_TRY(cudaMemcpyAsync(h->W.p, w_inv, nn * sizeof(double), cudaMemcpyHostToDevice, h->s));
    k_fwd_assemble<<<grid_for(nn), 256, 0, h->s>>>(h->W.p, h->Rprev.p, h->inv.A.p, h->n);
    SCATT_CUDA_TRY(cudaGetLastError());
    SCATT_COUNT_LAUNCH(1);
    SCATT_TRY(h->inv.run(true, h->s, "GpuForwardStepper::step"));
    SCATT_CUDA_TRY(cudaMemcpyAsync(h->Rprev.p, h->Rout.p, nn * sizeof(double), cudaMemcpyDeviceToDevice, h->s));
    SCATT_CUDA_TRY(cudaMemcpyAsync(rinv_out, h->Rout.p, nn * sizeof(double), cudaMemcpyDeviceToHost, h->s));
    SCATT_CUDA_TRY(cudaStreamSynchronize(h->s));
    if (max_asym_out) *max_asym_out = max_asym(rinv_out, h->n);
    return SCATT_OK;
}

// ------------------------------------------------------------- Sinv
int scatt_sinv_stepper_create(int device, int n_psi, int n_f, scatt_sinv_stepper** out) {
    if (!out || n_psi <= 0 || n_f < 0) {
        set_last_error("scatt_sinv_stepper_create: bad arguments");
        return SCATT_ERR_ARG;
    }
    *out = nullptr;
    auto* h = new scatt_sinv_stepper();
    int st = open_stepper(device, h);
    h->np = n_psi;
    h->nf = n_f;
    const size_t pf = (size_t)n_psi * std::max(1, n_f);
    if (st == SCATT_OK) st = h->B.alloc(pf);
    if (st == SCATT_OK) st = h->Bs.alloc(pf);
    if (st == SCATT_OK) st = h->Dinv.alloc(std::max(1, n_f));
    if (st == SCATT_OK) st = h->Sout.alloc((size_t)n_psi * n_psi);
    if (st == SCATT_OK) st = h->gm.alloc(1);
    if (st == SCATT_OK) st = h->inv.setup(n_psi, h->Sout.p);
    if (st != SCATT_OK) {
        close_stepper(h);
        return st;
    }
    *out = h;
    return SCATT_OK;
}

int scatt_sinv_stepper_destroy(scatt_sinv_stepper* h) {
    close_stepper(h);
    return SCATT_OK;
}

// Sinv = sym((A - B diag(Dinv) B^T)^-1); B and Dinv may be NULL (or n_f = 0)
// for the inverse-only variant (no exchange coupling, S = A).
int scatt_sinv_stepper_step(scatt_sinv_stepper* h, const double* A, const double* B, const double* dinv,
                            double* sinv_out, double* max_asym_out) {
    if (!h || !A || !sinv_out) return SCATT_ERR_ARG;
    SCATT_CUDA_TRY(cudaSetDevice(h->device));
    const int np = h->np, nf = h->nf;
    const size_t nn = (size_t)np * np;
    SCATT_CUDA_TRY(cudaMemcpyAsync(h->inv.A.p, A, nn * sizeof(double), cudaMemcpyHostToDevice, h->s));
    if (B && dinv && nf > 0) {
        const size_t pf = (size_t)np * nf;
        SCATT_CUDA_TRY(cudaMemcpyAsync(h->B.p, B, pf * sizeof(double), cudaMemcpyHostToDevice, h->s));
        SCATT_CUDA_TRY(cudaMemcpyAsync(h->Dinv.p, dinv, nf * sizeof(double), cudaMemcpyHostToDevice, h->s));
        k_scale_cols<<<grid_for(pf), 256, 0, h->s>>>(h->B.p, h->Dinv.p, h->Bs.p, np, nf);
        SCATT_CUDA_TRY(cudaGetLastError());
        SCATT_COUNT_LAUNCH(1);
        // S = A - Bs B^T (general product: A is the caller's and need not be symmetric)
        SCATT_TRY(gemm_one(h->gm, GemmEntry{h->Bs.p, h->B.p, h->inv.A.p, np, np, nf, np, np, np, -1.0, 1.0}, 0, 1,
                           h->s));
    }
    SCATT_TRY(h->inv.run(true, h->s, "GpuSinvStepper::step"));
    SCATT_CUDA_TRY(cudaMemcpyAsync(sinv_out, h->Sout.p, nn * sizeof(double), cudaMemcpyDeviceToHost, h->s));
    SCATT_CUDA_TRY(cudaStreamSynchronize(h->s));
    if (max_asym_out) *max_asym_out = max_asym(sinv_out, np);
    return SCATT_OK;
}

// ------------------------------------------------------------- back
int scatt_back_stepper_create(int device, int n_total, int n_psi, scatt_back_stepper** out) {
    if (!out || n_total <= 0 || n_psi <= 0 || n_psi > n_total) {
        set_last_error("scatt_back_stepper_create: bad arguments");
        return SCATT_ERR_ARG;
    }
    *out = nullptr;
    auto* h = new scatt_back_stepper();
    int st = open_stepper(device, h);
    h->nt = n_total;
    h->np = n_psi;
    h->nf = n_total - n_psi;
    const size_t nn = (size_t)n_total * n_total, nz = (size_t)n_total * n_psi;
    if (st == SCATT_OK) st = h->R.alloc(nn);
    if (st == SCATT_OK) st = h->W.alloc(nn);
    if (st == SCATT_OK) st = h->Z0.alloc(nz);
    if (st == SCATT_OK) st = h->Z1.alloc(nz);
    if (st == SCATT_OK) st = h->Y.alloc(nz);
    if (st == SCATT_OK) st = h->gm.alloc(1);
    if (st != SCATT_OK) {
        close_stepper(h);
        return st;
    }
    *out = h;
    return SCATT_OK;
}

int scatt_back_stepper_destroy(scatt_back_stepper* h) {
    close_stepper(h);
    return SCATT_OK;
}

int scatt_back_stepper_init(scatt_back_stepper* h, const double* Z) {
    if (!h || !Z) return SCATT_ERR_ARG;
    SCATT_CUDA_TRY(cudaSetDevice(h->device));
    SCATT_CUDA_TRY(cudaMemcpyAsync(h->Z0.p, Z, (size_t)h->nt * h->np * sizeof(double), cudaMemcpyHostToDevice,
                                   h->s));
    SCATT_CUDA_TRY(cudaStreamSynchronize(h->s));
    h->z_ready = true;
    return SCATT_OK;
}

// Z <- Rinv Z;  Y = W_inv Z;  psi = Y[0:n_psi, :], f = Y[n_psi:, :] (f_out may be NULL)
int scatt_back_stepper_step(scatt_back_stepper* h, const double* rinv, const double* w_inv, double* psi_out,
                            double* f_out) {
    if (!h || !rinv || !w_inv || !psi_out) return SCATT_ERR_ARG;
    if (!h->z_ready) {
        set_last_error("GpuBackStepper::step: call scatt_back_stepper_init first");
        return SCATT_ERR_STATE;
    }
    SCATT_CUDA_TRY(cudaSetDevice(h->device));
    const int nt = h->nt, np = h->np, nf = h->nf;
    const size_t nn = (size_t)nt * nt;
    SCATT_CUDA_TRY(cudaMemcpyAsync(h->R.p, rinv, nn * sizeof(double), cudaMemcpyHostToDevice, h->s));
    SCATT_CUDA_TRY(cudaMemcpyAsync(h->W.p, w_inv, nn * sizeof(double), cudaMemcpyHostToDevice, h->s));
    SCATT_TRY(gemm_one(h->gm, GemmEntry{h->R.p, h->Z0.p, h->Z1.p, nt, np, nt, nt, nt, nt, 1.0, 0.0}, 0, 0, h->s));
    SCATT_TRY(gemm_one(h->gm, GemmEntry{h->W.p, h->Z1.p, h->Y.p, nt, np, nt, nt, nt, nt, 1.0, 0.0}, 0, 0, h->s));
    std::swap(h->Z0.p, h->Z1.p);
    SCATT_CUDA_TRY(cudaMemcpy2DAsync(psi_out, np * sizeof(double), h->Y.p, nt * sizeof(double), np * sizeof(double),
                                     np, cudaMemcpyDeviceToHost, h->s));
    if (f_out && nf > 0)
        SCATT_CUDA_TRY(cudaMemcpy2DAsync(f_out, nf * sizeof(double), h->Y.p + np, nt * sizeof(double),
                                         nf * sizeof(double), np, cudaMemcpyDeviceToHost, h->s));
    SCATT_CUDA_TRY(cudaStreamSynchronize(h->s));
    return SCATT_OK;
}

int scatt_back_stepper_get_z(scatt_back_stepper* h, double* Z_out) {
    if (!h || !Z_out) return SCATT_ERR_ARG;
    SCATT_CUDA_TRY(cudaSetDevice(h->device));
    SCATT_CUDA_TRY(cudaMemcpyAsync(Z_out, h->Z0.p, (size_t)h->nt * h->np * sizeof(double), cudaMemcpyDeviceToHost,
                                   h->s));
    SCATT_CUDA_TRY(cudaStreamSynchronize(h->s));
    return SCATT_OK;
}

}  // extern "C"
