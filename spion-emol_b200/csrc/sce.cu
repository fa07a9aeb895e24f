// sce.cu -- the single-centre expansion of the preprocessing step
// (preprocessing/src/sce/SCE.hpp:122-266, project) on the DMMA tensor
// cores: F_lm(r) = int F(r, Omega) Y^R_lm(Omega) dOmega from samples of F
// on the grid of preprocessing/src/angular/Grid.hpp (n_theta = Lmax + 1
// Gauss-Legendre nodes in cos(theta), ascending; n_phi = 2 (Lmax + 1)
// nodes phi_j = 2 pi j / n_phi).
//
// The reference factors the projection into a Fourier step in phi and a
// Legendre step in theta, per radial point.  Here both steps are GEMMs over
// a chunk of R radial points:
//
//   1. A_m, B_m (m = 0 .. Lmax): C1 = X^T T, with X the chunk's samples
//      (n_phi x R n_theta, rows contiguous) and T = [cos(m phi_j) | sin(m phi_j)]
//      (n_phi x 2 Lmax + 1): one GEMM of M = R n_theta, N = 2 Lmax + 1,
//      K = n_phi.  Column m of C1, read as an n_theta x R matrix, is A_m.
//   2. For every m: Q_m = P_m A_m with P_m[l - m, i] = c_m dphi w_i S_lm(theta_i)
//      (c_0 = 1, c_m = sqrt 2), and the same for B_m: 2 Lmax + 1 GEMMs of
//      (Lmax + 1 - m) x R x n_theta in one batched launch.
//   3. A gather kernel places Q's rows at the channels l^2 + l +- m.
//
// S_lm is the normalised associated Legendre function without the
// Condon-Shortley phase (angular/Legendre.hpp:11-31), by the standard
// recurrence of Holmes and Featherstone (2002); the Gauss-Legendre nodes by
// Newton's iteration on the Legendre recurrence.  Both are host-side tables.
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "common.cuh"
#include "devbuf.cuh"

namespace scatt {
namespace {

constexpr double SCE_PI = 3.14159265358979323846;

// Legendre P_n(z) and P_{n-1}(z) by the three-term recurrence, n >= 1.
void legendre_pair(int n, double z, double& pn, double& pm) {
    double p0 = 1.0, p1 = z;
    for (int k = 2; k <= n; ++k) {
        const double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
        p0 = p1;
        p1 = p2;
    }
    pn = p1;
    pm = p0;
}

// Gauss-Legendre nodes (ascending) and weights on [-1, 1], n >= 1: Newton's
// iteration on P_n from cos(pi (i + 3/4) / (n + 1/2)), P_n' = n (z P_n - P_{n-1}) / (z^2 - 1),
// w = 2 / ((1 - z^2) P_n'^2); the negative half by symmetry.
void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w) {
    x.assign(n, 0.0);
    w.assign(n, 0.0);
    for (int i = 0; i < (n + 1) / 2; ++i) {
        double z = std::cos(SCE_PI * (i + 0.75) / (n + 0.5)), pn, pm;
        for (int it = 0; it < 100; ++it) {
            legendre_pair(n, z, pn, pm);
            const double dz = pn / (n * (z * pn - pm) / (z * z - 1.0));
            z -= dz;
            if (std::fabs(dz) < 1e-16) break;
        }
        legendre_pair(n, z, pn, pm);
        const double dp = n * (z * pn - pm) / (z * z - 1.0);
        const double wi = 2.0 / ((1.0 - z * z) * dp * dp);
        x[n - 1 - i] = z;                                   // the largest node first
        x[i] = -z;
        w[n - 1 - i] = wi;
        w[i] = wi;
    }
    if (n % 2 == 1) x[n / 2] = 0.0;
}

// S[(l (L + 1) + m) n + i] = S_{l,m}(theta_i) for m <= l <= L.
std::vector<double> s_table(int L, const std::vector<double>& cth) {
    const int n = (int)cth.size();
    std::vector<double> S((size_t)(L + 1) * (L + 1) * n, 0.0);
    auto at = [&](int l, int m, int i) -> double& { return S[((size_t)l * (L + 1) + m) * n + i]; };
    for (int i = 0; i < n; ++i) {
        const double c = cth[i], s = std::sqrt(std::max(0.0, 1.0 - c * c));
        double smm = 1.0 / std::sqrt(4.0 * SCE_PI);
        for (int m = 0; m <= L; ++m) {
            if (m > 0) smm *= std::sqrt((2.0 * m + 1.0) / (2.0 * m)) * s;
            at(m, m, i) = smm;
            if (m + 1 <= L) at(m + 1, m, i) = std::sqrt(2.0 * m + 3.0) * c * smm;
            for (int k = m + 2; k <= L; ++k) {
                const double a = std::sqrt((4.0 * k * k - 1.0) / ((double)k * k - (double)m * m));
                const double b = std::sqrt(((double)(k - 1) * (k - 1) - (double)m * m) / (4.0 * (k - 1) * (k - 1) - 1.0));
                at(k, m, i) = a * (c * at(k - 1, m, i) - b * at(k - 2, m, i));
            }
        }
    }
    return S;
}

// out[ch R + k] = Q rows: channel l^2 + l + m (m >= 0) from the cos block of m,
// l^2 + l - m from the sin block; block m has L + 1 - m rows, ld L + 1 - m.
__global__ void k_sce_gather(const double* __restrict__ Q, const long* __restrict__ off_c,
                             const long* __restrict__ off_s, int L, int R, double* __restrict__ out) {
    const long n_lm = (long)(L + 1) * (L + 1);
    const long total = n_lm * R;
    for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total; idx += (long)gridDim.x * blockDim.x) {
        const int k = (int)(idx % R);
        const int ch = (int)(idx / R);
        const int l = (int)sqrt((double)ch + 0.5);
        const int m = ch - l * l - l;
        const int am = m < 0 ? -m : m;
        const long base = m < 0 ? off_s[am] : off_c[am];
        out[idx] = Q[base + (l - am) + (long)k * (L + 1 - am)];
    }
}

struct SceStream {
    cudaStream_t s = nullptr;
    ~SceStream() { if (s) cudaStreamDestroy(s); }
};

}  // namespace
}  // namespace scatt

using namespace scatt;

extern "C" {

int scatt_sce_grid(int Lmax, double* cos_theta, double* weights, double* phi) {
    if (Lmax < 0 || !cos_theta || !weights || !phi) {
        set_last_error("scatt_sce_grid: need Lmax >= 0 and the three buffers");
        return SCATT_ERR_ARG;
    }
    std::vector<double> x, w;
    gauss_legendre(Lmax + 1, x, w);
    std::copy(x.begin(), x.end(), cos_theta);
    std::copy(w.begin(), w.end(), weights);
    const int n_phi = 2 * (Lmax + 1);
    for (int j = 0; j < n_phi; ++j) phi[j] = 2.0 * SCE_PI * j / n_phi;
    return SCATT_OK;
}

int scatt_sce_project(int Lmax, int Nr, int chunk, const double* samples, double* F_lm) {
    if (Lmax < 0 || Nr < 1 || !samples || !F_lm) {
        set_last_error("scatt_sce_project: need Lmax >= 0, Nr >= 1 and the buffers");
        return SCATT_ERR_ARG;
    }
    SCATT_TRY(require_device());
    const int L = Lmax, nT = L + 1, nP = 2 * (L + 1), nM = 2 * L + 1;
    const long n_lm = (long)(L + 1) * (L + 1);
    // radial points per device pass: samples, C1, Q and the gathered rows within 64 Mi doubles
    const long per_pt = (long)nT * nP + (long)nT * nM + 2 * n_lm;
    int R = chunk > 0 ? chunk : (int)std::max<long>(1, (64L << 20) / per_pt);
    R = std::min(R, Nr);
    if ((long)R * nT > (1L << 30)) R = (int)std::max<long>(1, (1L << 30) / nT);
    // ---- host tables: grid, trig table T (n_phi x nM), P_m blocks
    std::vector<double> x, w;
    gauss_legendre(nT, x, w);
    const std::vector<double> S = s_table(L, x);
    const double dphi = 2.0 * SCE_PI / nP;
    std::vector<double> T((size_t)nP * nM);
    for (int j = 0; j < nP; ++j) {
        const double ph = 2.0 * SCE_PI * j / nP;
        for (int m = 0; m <= L; ++m) T[j + (size_t)m * nP] = std::cos(m * ph);
        for (int m = 1; m <= L; ++m) T[j + (size_t)(L + m) * nP] = std::sin(m * ph);
    }
    std::vector<long> poff(L + 1);
    long ptot = 0;
    for (int m = 0; m <= L; ++m) { poff[m] = ptot; ptot += (long)(L + 1 - m) * nT; }
    std::vector<double> P(ptot);
    for (int m = 0; m <= L; ++m) {
        const int rows = L + 1 - m;
        const double c = (m == 0 ? 1.0 : std::sqrt(2.0)) * dphi;
        for (int i = 0; i < nT; ++i)
            for (int l = m; l <= L; ++l)
                P[poff[m] + (l - m) + (long)i * rows] = c * w[i] * S[((size_t)l * (L + 1) + m) * nT + i];
    }
    // Q blocks: cos block of m, then sin blocks, R columns each (offsets for a full chunk;
    // a shorter last chunk packs them tighter with the same formula)
    auto q_offsets = [&](int Rc, std::vector<long>& oc, std::vector<long>& os) {
        oc.assign(L + 1, 0);
        os.assign(L + 1, 0);
        long o = 0;
        for (int m = 0; m <= L; ++m) { oc[m] = o; o += (long)(L + 1 - m) * Rc; }
        for (int m = 1; m <= L; ++m) { os[m] = o; o += (long)(L + 1 - m) * Rc; }
        return o;
    };
    std::vector<long> oc, os;
    const long qtot = q_offsets(R, oc, os);
    SceStream st;
    SCATT_CUDA_TRY(cudaStreamCreateWithFlags(&st.s, cudaStreamNonBlocking));
    const cudaStream_t s = st.s;
    DevBuf<double> dX, dT, dP, dC1, dQ, dOut;
    DevBuf<long> doc, dos;
    DevBuf<GemmEntry> de1, de2;
    SCATT_TRY(dX.alloc((size_t)R * nT * nP));
    SCATT_TRY(dC1.alloc((size_t)R * nT * nM));
    SCATT_TRY(dQ.alloc((size_t)qtot));
    SCATT_TRY(dOut.alloc((size_t)n_lm * R));
    SCATT_TRY(dT.upload(T, s));
    SCATT_TRY(dP.upload(P, s));
    SCATT_TRY(doc.alloc(L + 1));
    SCATT_TRY(dos.alloc(L + 1));
    SCATT_TRY(de1.alloc(1));
    SCATT_TRY(de2.alloc(nM));
    std::vector<GemmEntry> e2(nM);
    for (int c0 = 0; c0 < Nr; c0 += R) {
        const int Rc = std::min(R, Nr - c0);
        const long M1 = (long)Rc * nT;
        q_offsets(Rc, oc, os);
        const GemmEntry e1{dX.p, dT.p, dC1.p, (int)M1, nM, nP, nP, nP, (int)M1, 1.0, 0.0};
        for (int m = 0; m <= L; ++m)
            e2[m] = GemmEntry{dP.p + poff[m], dC1.p + (size_t)m * M1, dQ.p + oc[m], L + 1 - m, Rc, nT,
                              L + 1 - m, nT, L + 1 - m, 1.0, 0.0};
        for (int m = 1; m <= L; ++m)
            e2[L + m] = GemmEntry{dP.p + poff[m], dC1.p + (size_t)(L + m) * M1, dQ.p + os[m], L + 1 - m, Rc, nT,
                                  L + 1 - m, nT, L + 1 - m, 1.0, 0.0};
        SCATT_CUDA_TRY(cudaMemcpyAsync(de1.p, &e1, sizeof(GemmEntry), cudaMemcpyHostToDevice, s));
        SCATT_CUDA_TRY(cudaMemcpyAsync(de2.p, e2.data(), nM * sizeof(GemmEntry), cudaMemcpyHostToDevice, s));
        SCATT_CUDA_TRY(cudaMemcpyAsync(doc.p, oc.data(), (L + 1) * sizeof(long), cudaMemcpyHostToDevice, s));
        SCATT_CUDA_TRY(cudaMemcpyAsync(dos.p, os.data(), (L + 1) * sizeof(long), cudaMemcpyHostToDevice, s));
        SCATT_CUDA_TRY(cudaMemcpyAsync(dX.p, samples + (size_t)c0 * nT * nP, (size_t)Rc * nT * nP * sizeof(double),
                                       cudaMemcpyHostToDevice, s));
        SCATT_TRY(gemm_batched(de1.p, 1, (int)M1, nM, 1, 0, s));             // A_m, B_m of every (r, theta)
        SCATT_TRY(gemm_batched(de2.p, nM, L + 1, Rc, 0, 0, s));              // the Legendre step per m
        const long tot = n_lm * Rc;
        const int grid = (int)std::max<long>(1, std::min<long>((tot + 255) / 256, 148L * 8));
        k_sce_gather<<<grid, 256, 0, s>>>(dQ.p, doc.p, dos.p, L, Rc, dOut.p);
        SCATT_COUNT_LAUNCH(1);
        SCATT_CUDA_TRY(cudaGetLastError());
        SCATT_CUDA_TRY(cudaMemcpy2DAsync(F_lm + c0, (size_t)Nr * sizeof(double), dOut.p, (size_t)Rc * sizeof(double),
                                         (size_t)Rc * sizeof(double), (size_t)n_lm, cudaMemcpyDeviceToHost, s));
        // the host tables of the next chunk overwrite e1 / e2 / oc / os: finish this one first
        SCATT_CUDA_TRY(cudaStreamSynchronize(s));
    }
    return SCATT_OK;
}

}  // extern "C"
