// cc_dipole.cu -- the continuum-continuum dipole, the consumer of the psi
// store (postprocessing/two_photon_delay/cc_dipole/src/CCDipole.cpp:294-334,
// in the range-accumulating form of include/CCDipole.hpp): for one final
// state kappa and n_nu intermediate states nu,
//
//   cc_nu[beta, alpha] = sum_i w_i r_i sum_{mu, mu'} psi_kappa(i)[mu, beta] A^q[mu, mu'] psi_nu(i)[mu', alpha]
//
// over the radial points ir0 .. ir0 + n_pts - 1, with r_i = (ir0 + i + 1) dr
// (r_min = dr, CCDipole.cpp:236), w_i the Simpson weights of the window
// (:100-122) and A^q = sqrt(4 pi / 3) gaunt_real(l_mu, m_mu, 1, q, l_mu', m_mu')
// (:135-160), which has at most four non-zeros per row.  Length gauge, as
// the reference (:294-303).
//
// Points stream through the device in chunks.  A chunk of psi_kappa is
// restacked once into V_X (P n_mu rows x n_mu columns; row i n_mu + mu holds
// psi_kappa(i)[mu, :]); for each nu the sparse angular product lands in V_T
// the same way (row i n_mu + mu holds w_i r_i (A^q psi_nu(i))[mu, :]).  The
// chunk's share of cc_nu is then the single contraction V_X^T V_T over
// K = P n_mu: a DMMA GEMM split along K into batched pieces, so that enough
// CTAs cover the SMs, whose partial products are summed in a fixed order.
#include <algorithm>
#include <string>
#include <vector>

#include "angular.hpp"
#include "common.cuh"
#include "devbuf.cuh"

namespace scatt {
namespace {

constexpr int CC_TPB = 256;

// V[(i n_mu + mu) + b (P n_mu)] = X[i ld^2 + mu + b ld]
__global__ void k_cc_stack(const double* __restrict__ X, int ld, int n_mu, int P, double* __restrict__ V) {
    const long rows = (long)P * n_mu, total = rows * n_mu;
    for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total; idx += (long)gridDim.x * blockDim.x) {
        const long row = idx % rows;
        const int b = (int)(idx / rows);
        const int i = (int)(row / n_mu), mu = (int)(row - (long)i * n_mu);
        V[idx] = X[(size_t)i * ld * ld + mu + (size_t)b * ld];
    }
}

// V[(i n_mu + mu) + a (P n_mu)] = wr[i] sum_k av[k] X[i ld^2 + ci[k] + a ld], k in [rp[mu], rp[mu + 1])
__global__ void k_cc_apply(const double* __restrict__ X, int ld, int n_mu, int P, const int* __restrict__ rp,
                           const int* __restrict__ ci, const double* __restrict__ av,
                           const double* __restrict__ wr, double* __restrict__ V) {
    const long rows = (long)P * n_mu, total = rows * n_mu;
    for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total; idx += (long)gridDim.x * blockDim.x) {
        const long row = idx % rows;
        const int a = (int)(idx / rows);
        const int i = (int)(row / n_mu), mu = (int)(row - (long)i * n_mu);
        const double* x = X + (size_t)i * ld * ld + (size_t)a * ld;
        double s = 0.0;
        for (int k = rp[mu]; k < rp[mu + 1]; ++k) s = fma(av[k], x[ci[k]], s);
        V[idx] = wr[i] * s;
    }
}

// cc[idx] += sum_s part[s nn + idx], s = 0 .. S - 1 in order
__global__ void k_cc_reduce(const double* __restrict__ part, int S, int nn, double* __restrict__ cc) {
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < nn; idx += gridDim.x * blockDim.x) {
        double s = cc[idx];
        for (int k = 0; k < S; ++k) s += part[(size_t)k * nn + idx];
        cc[idx] = s;
    }
}

int grid_for(long total) { return (int)std::max<long>(1, std::min<long>((total + CC_TPB - 1) / CC_TPB, 148L * 8)); }

// Simpson weights of an n-point window of step h (CCDipole.cpp:100-122):
// composite 1/3 rule for odd n; for even n the 1/3 rule on the first n - 3
// points and the 3/8 rule on the last four.
std::vector<double> simpson_weights(int n, double h) {
    std::vector<double> w(n, 0.0);
    if (n % 2 == 1) {
        w[0] = w[n - 1] = h / 3.0;
        for (int i = 1; i < n - 1; ++i) w[i] = ((i & 1) ? 4.0 : 2.0) * h / 3.0;
        return w;
    }
    const int n13 = n - 3;
    if (n13 >= 2) {
        w[0] += h / 3.0;
        w[n13 - 1] += h / 3.0;
        for (int i = 1; i < n13 - 1; ++i) w[i] += ((i & 1) ? 4.0 : 2.0) * h / 3.0;
    }
    const double s38 = 3.0 * h / 8.0;
    const int j = n - 4;
    w[j] += s38;
    w[j + 1] += 3.0 * s38;
    w[j + 2] += 3.0 * s38;
    w[j + 3] += s38;
    return w;
}

struct CcStream {
    cudaStream_t s = nullptr;
    ~CcStream() { if (s) cudaStreamDestroy(s); }
};

}  // namespace
}  // namespace scatt

using namespace scatt;

extern "C" int scatt_cc_dipole(int n_mu, int ld, int n_pts, int ir0, double dr, int q, const double* psi_kappa,
                               int n_nu, const double* psi_nu, double* cc) {
    if (n_mu < 1 || ld < n_mu || ir0 < 0 || !(dr > 0.0) || q < -1 || q > 1 || n_nu < 1 || !psi_kappa ||
        !psi_nu || !cc) {
        set_last_error("scatt_cc_dipole: need n_mu >= 1, ld >= n_mu, ir0 >= 0, dr > 0, q in {-1, 0, 1}, "
                       "n_nu >= 1 and the buffers");
        return SCATT_ERR_ARG;
    }
    if (n_pts < 5) {
        set_last_error("cc_dipole: too few overlapping radial points (" + std::to_string(n_pts) + " < 5)");
        return SCATT_ERR_ARG;
    }
    SCATT_TRY(require_device());
    // angular table A^q, one CSR row per channel mu
    std::vector<int> rp(n_mu + 1, 0), ci;
    std::vector<double> av;
    for (int mu = 0; mu < n_mu; ++mu) {
        int l1, m1;
        idx_to_lm(mu, l1, m1);
        for (int nu = 0; nu < n_mu; ++nu) {
            int l2, m2;
            idx_to_lm(nu, l2, m2);
            if (std::abs(l1 - l2) != 1) continue;
            const double v = angular_dipole(l1, m1, q, l2, m2);
            if (v != 0.0) {
                ci.push_back(nu);
                av.push_back(v);
            }
        }
        rp[mu + 1] = (int)ci.size();
    }
    if (ci.empty()) { ci.push_back(0); av.push_back(0.0); }
    std::vector<double> wr = simpson_weights(n_pts, dr);
    for (int i = 0; i < n_pts; ++i) wr[i] *= (double)(ir0 + i + 1) * dr;
    // chunk of points: the raw psi and the two stacks of a chunk in at most 64 Mi doubles (512 MB)
    const size_t ld2 = (size_t)ld * ld, nn = (size_t)n_mu * n_mu;
    const size_t per_pt = 2 * ld2 + 2 * nn;
    const int P = (int)std::max<size_t>(1, std::min<size_t>((size_t)n_pts, (size_t(64) << 20) / per_pt));
    // split of K = P n_mu: enough pieces that the GEMM covers the SMs four times over
    const int tiles = ((n_mu + 127) / 128) * ((n_mu + 63) / 64);
    const long Kmax = (long)P * n_mu;
    const int S_want = std::max(1, (4 * 148 + tiles - 1) / tiles);
    long Kc = std::max<long>(256, (Kmax + S_want - 1) / S_want);
    Kc = (Kc + 31) / 32 * 32;
    const int S_max = (int)((Kmax + Kc - 1) / Kc);
    CcStream st;
    SCATT_CUDA_TRY(cudaStreamCreateWithFlags(&st.s, cudaStreamNonBlocking));
    const cudaStream_t s = st.s;
    DevBuf<double> dXk, dXn, dVX, dVT, dpart, dcc, dwr, dav;
    DevBuf<int> drp, dci;
    DevBuf<GemmEntry> dent;
    SCATT_TRY(dXk.alloc((size_t)P * ld2));
    SCATT_TRY(dXn.alloc((size_t)P * ld2));
    SCATT_TRY(dVX.alloc((size_t)P * nn));
    SCATT_TRY(dVT.alloc((size_t)P * nn));
    SCATT_TRY(dpart.alloc((size_t)S_max * nn));
    SCATT_TRY(dcc.alloc((size_t)n_nu * nn));
    SCATT_TRY(dent.alloc(S_max));
    SCATT_TRY(dwr.upload(wr, s));
    SCATT_TRY(drp.upload(rp, s));
    SCATT_TRY(dci.upload(ci, s));
    SCATT_TRY(dav.upload(av, s));
    SCATT_CUDA_TRY(cudaMemsetAsync(dcc.p, 0, (size_t)n_nu * nn * sizeof(double), s));
    std::vector<GemmEntry> ent(S_max);
    for (int c0 = 0; c0 < n_pts; c0 += P) {
        const int Pc = std::min(P, n_pts - c0);
        const long K = (long)Pc * n_mu;
        const int S = (int)((K + Kc - 1) / Kc);
        for (int k = 0; k < S; ++k) {
            const long k0 = (long)k * Kc;
            ent[k] = GemmEntry{dVX.p + k0, dVT.p + k0, dpart.p + (size_t)k * nn, n_mu, n_mu,
                               (int)std::min<long>(Kc, K - k0), (int)K, (int)K, n_mu, 1.0, 0.0};
        }
        SCATT_CUDA_TRY(cudaMemcpyAsync(dent.p, ent.data(), S * sizeof(GemmEntry), cudaMemcpyHostToDevice, s));
        SCATT_CUDA_TRY(cudaMemcpyAsync(dXk.p, psi_kappa + (size_t)c0 * ld2, (size_t)Pc * ld2 * sizeof(double),
                                       cudaMemcpyHostToDevice, s));
        k_cc_stack<<<grid_for(K * n_mu), CC_TPB, 0, s>>>(dXk.p, ld, n_mu, Pc, dVX.p);
        SCATT_COUNT_LAUNCH(1);
        for (int v = 0; v < n_nu; ++v) {
            SCATT_CUDA_TRY(cudaMemcpyAsync(dXn.p, psi_nu + ((size_t)v * n_pts + c0) * ld2,
                                           (size_t)Pc * ld2 * sizeof(double), cudaMemcpyHostToDevice, s));
            k_cc_apply<<<grid_for(K * n_mu), CC_TPB, 0, s>>>(dXn.p, ld, n_mu, Pc, drp.p, dci.p, dav.p, dwr.p + c0,
                                                             dVT.p);
            SCATT_COUNT_LAUNCH(1);
            SCATT_TRY(gemm_batched(dent.p, S, n_mu, n_mu, 1, 0, s));
            k_cc_reduce<<<grid_for((long)nn), CC_TPB, 0, s>>>(dpart.p, S, (int)nn, dcc.p + (size_t)v * nn);
            SCATT_COUNT_LAUNCH(1);
        }
        SCATT_CUDA_TRY(cudaGetLastError());
    }
    SCATT_CUDA_TRY(cudaMemcpyAsync(cc, dcc.p, (size_t)n_nu * nn * sizeof(double), cudaMemcpyDeviceToHost, s));
    SCATT_CUDA_TRY(cudaStreamSynchronize(s));
    return SCATT_OK;
}
