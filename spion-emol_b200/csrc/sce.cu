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

// out[f][ch R + k] = Q rows of function f: channel l^2 + l + m (m >= 0) from
// the cos block of m, l^2 + l - m from the sin block; block m has L + 1 - m
// rows, ld L + 1 - m; function f's blocks start at f qstride.
__global__ void k_sce_gather(const double* __restrict__ Q, long qstride, const long* __restrict__ off_c,
                             const long* __restrict__ off_s, int L, int R, double* __restrict__ out) {
    const long n_lm = (long)(L + 1) * (L + 1);
    const long total = n_lm * R;
    const double* q = Q + (size_t)blockIdx.y * qstride;
    double* o = out + (size_t)blockIdx.y * total;
    for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total; idx += (long)gridDim.x * blockDim.x) {
        const int k = (int)(idx % R);
        const int ch = (int)(idx / R);
        const int l = (int)sqrt((double)ch + 0.5);
        const int m = ch - l * l - l;
        const int am = m < 0 ? -m : m;
        const long base = m < 0 ? off_s[am] : off_c[am];
        o[idx] = q[base + (l - am) + (long)k * (L + 1 - am)];
    }
}

struct SceStream {
    cudaStream_t s = nullptr;
    ~SceStream() { if (s) cudaStreamDestroy(s); }
};

// The projection of n_fn functions at a time over chunks of up to R radial
// points: host tables (trig table T, Legendre blocks P_m) on the device,
// scratch for the Fourier products C1 and the Legendre products Q.
struct SceProjector {
    int L = 0, nT = 0, nP = 0, nM = 0, n_fn = 1, R = 1;
    long n_lm = 0;
    std::vector<double> x, w;                 // the Gauss-Legendre nodes and weights
    std::vector<long> poff, oc, os;
    std::vector<GemmEntry> e1, e2;
    DevBuf<double> T, P, C1, Q;
    DevBuf<long> doc, dos;
    DevBuf<GemmEntry> de1, de2;

    // Q blocks of one function for a chunk of Rc points: cos blocks, then sin
    long q_offsets(int Rc) {
        oc.assign(L + 1, 0);
        os.assign(L + 1, 0);
        long o = 0;
        for (int m = 0; m <= L; ++m) { oc[m] = o; o += (long)(L + 1 - m) * Rc; }
        for (int m = 1; m <= L; ++m) { os[m] = o; o += (long)(L + 1 - m) * Rc; }
        return o;
    }

    int init(int Lmax, int nfn, int Rmax, cudaStream_t s) {
        L = Lmax; nT = L + 1; nP = 2 * (L + 1); nM = 2 * L + 1; n_fn = nfn; R = Rmax;
        n_lm = (long)(L + 1) * (L + 1);
        gauss_legendre(nT, x, w);
        const std::vector<double> S = s_table(L, x);
        const double dphi = 2.0 * SCE_PI / nP;
        std::vector<double> Th((size_t)nP * nM);
        for (int j = 0; j < nP; ++j) {
            const double ph = 2.0 * SCE_PI * j / nP;
            for (int m = 0; m <= L; ++m) Th[j + (size_t)m * nP] = std::cos(m * ph);
            for (int m = 1; m <= L; ++m) Th[j + (size_t)(L + m) * nP] = std::sin(m * ph);
        }
        poff.assign(L + 1, 0);
        long ptot = 0;
        for (int m = 0; m <= L; ++m) { poff[m] = ptot; ptot += (long)(L + 1 - m) * nT; }
        std::vector<double> Ph(ptot);
        for (int m = 0; m <= L; ++m) {
            const int rows = L + 1 - m;
            const double c = (m == 0 ? 1.0 : std::sqrt(2.0)) * dphi;
            for (int i = 0; i < nT; ++i)
                for (int l = m; l <= L; ++l)
                    Ph[poff[m] + (l - m) + (long)i * rows] = c * w[i] * S[((size_t)l * (L + 1) + m) * nT + i];
        }
        SCATT_TRY(T.upload(Th, s));
        SCATT_TRY(P.upload(Ph, s));
        SCATT_TRY(C1.alloc((size_t)n_fn * R * nT * nM));
        SCATT_TRY(Q.alloc((size_t)n_fn * q_offsets(R)));
        SCATT_TRY(doc.alloc(L + 1));
        SCATT_TRY(dos.alloc(L + 1));
        SCATT_TRY(de1.alloc(n_fn));
        SCATT_TRY(de2.alloc((size_t)n_fn * nM));
        e1.resize(n_fn);
        e2.resize((size_t)n_fn * nM);
        // the host tables above are pageable: their copies are staged before the call returns
        return SCATT_CUDA_TRY_RET(cudaStreamSynchronize(s));
    }

    // X: the samples of function f at X + f fstride, [Rc][n_theta][n_phi];
    // out: [n_fn][n_lm][Rc].  Returns once the work is queued on s; the
    // caller synchronises before the next run (the entry tables are reused).
    int run(const double* X, long fstride, int Rc, double* out, cudaStream_t s) {
        const long M1 = (long)Rc * nT;
        const long qs = q_offsets(Rc);
        for (int f = 0; f < n_fn; ++f) {
            double* c1 = C1.p + (size_t)f * M1 * nM;
            e1[f] = GemmEntry{X + (size_t)f * fstride, T.p, c1, (int)M1, nM, nP, nP, nP, (int)M1, 1.0, 0.0};
            for (int m = 0; m <= L; ++m)
                e2[(size_t)f * nM + m] = GemmEntry{P.p + poff[m], c1 + (size_t)m * M1, Q.p + f * qs + oc[m], L + 1 - m,
                                                   Rc, nT, L + 1 - m, nT, L + 1 - m, 1.0, 0.0};
            for (int m = 1; m <= L; ++m)
                e2[(size_t)f * nM + L + m] = GemmEntry{P.p + poff[m], c1 + (size_t)(L + m) * M1, Q.p + f * qs + os[m],
                                                       L + 1 - m, Rc, nT, L + 1 - m, nT, L + 1 - m, 1.0, 0.0};
        }
        SCATT_CUDA_TRY(cudaMemcpyAsync(de1.p, e1.data(), n_fn * sizeof(GemmEntry), cudaMemcpyHostToDevice, s));
        SCATT_CUDA_TRY(cudaMemcpyAsync(de2.p, e2.data(), e2.size() * sizeof(GemmEntry), cudaMemcpyHostToDevice, s));
        SCATT_CUDA_TRY(cudaMemcpyAsync(doc.p, oc.data(), (L + 1) * sizeof(long), cudaMemcpyHostToDevice, s));
        SCATT_CUDA_TRY(cudaMemcpyAsync(dos.p, os.data(), (L + 1) * sizeof(long), cudaMemcpyHostToDevice, s));
        SCATT_TRY(gemm_batched(de1.p, n_fn, (int)M1, nM, 1, 0, s));          // A_m, B_m of every (r, theta)
        SCATT_TRY(gemm_batched(de2.p, n_fn * nM, L + 1, Rc, 0, 0, s));       // the Legendre step per m
        const long tot = n_lm * Rc;
        const dim3 grid((unsigned)std::max<long>(1, std::min<long>((tot + 255) / 256, 148L * 8)), (unsigned)n_fn);
        k_sce_gather<<<grid, 256, 0, s>>>(Q.p, qs, doc.p, dos.p, L, Rc, out);
        SCATT_COUNT_LAUNCH(1);
        return SCATT_CUDA_TRY_RET(cudaGetLastError());
    }
};

// ---- Gaussian basis (MoldenBasis.hpp:48-229) on the grid's points

struct ShellDev {
    double cx, cy, cz;
    int l, nprim, off, ao0;   // primitives [off, off + nprim) of exps / ct; first AO index
};

__device__ __forceinline__ int molden_m(int l, int idx) {
    if (l == 0) return 0;
    if (l == 1) return idx == 0 ? 1 : (idx == 1 ? -1 : 0);
    if (idx == 0) return 0;
    const int half = (idx + 1) / 2;
    return (idx & 1) ? half : -half;
}

// S_{l,m} (no Condon-Shortley phase) from cos / sin of theta, 0 <= m <= l
__device__ double s_lm(int l, int m, double c, double s) {
    double smm = 0.28209479177387814347;            // 1 / sqrt(4 pi)
    for (int k = 1; k <= m; ++k) smm *= sqrt((2.0 * k + 1.0) / (2.0 * k)) * s;
    if (l == m) return smm;
    double a2 = smm, a1 = sqrt(2.0 * m + 3.0) * c * smm;
    for (int k = m + 2; k <= l; ++k) {
        const double a = sqrt((4.0 * k * k - 1.0) / ((double)k * k - (double)m * m));
        const double b = sqrt(((double)(k - 1) * (k - 1) - (double)m * m) / (4.0 * (k - 1) * (k - 1) - 1.0));
        const double t = a * (c * a1 - b * a2);
        a2 = a1;
        a1 = t;
    }
    return a1;
}

// Phi[mu + p nbf] = chi_mu at point p = (k, a): origin + r_k dir_a, r_k = r0 + (k0 + k) dr
__global__ void k_ao_eval(const ShellDev* __restrict__ sh, int n_shell, const double* __restrict__ exps,
                          const double* __restrict__ ct, const double* __restrict__ dir, int n_dir, int Pc,
                          double ox, double oy, double oz, double r0, double dr, int k0, int nbf,
                          double* __restrict__ Phi) {
    const long total = (long)Pc * n_shell;
    for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total; idx += (long)gridDim.x * blockDim.x) {
        const int si = (int)(idx % n_shell);
        const long p = idx / n_shell;
        const int k = (int)(p / n_dir), a = (int)(p - (long)k * n_dir);
        const double r = r0 + (k0 + k) * dr;
        const ShellDev S = sh[si];
        const double dx = ox + r * dir[3 * a] - S.cx, dy = oy + r * dir[3 * a + 1] - S.cy,
                     dz = oz + r * dir[3 * a + 2] - S.cz;
        const double r2 = dx * dx + dy * dy + dz * dz, rr = sqrt(r2);
        double rad = 0.0;
        for (int q = 0; q < S.nprim; ++q) rad += ct[S.off + q] * exp(-exps[S.off + q] * r2);
        double* out = Phi + (size_t)p * nbf + S.ao0;
        const int ncomp = S.l == 0 ? 1 : 2 * S.l + 1;
        if (rr < 1e-300) {
            for (int q = 0; q < ncomp; ++q) out[q] = (S.l == 0) ? 0.28209479177387814347 * rad : 0.0;
            continue;
        }
        const double c = fmin(1.0, fmax(-1.0, dz / rr));
        const double rxy = sqrt(dx * dx + dy * dy), s = rxy / rr;
        const double cp = rxy > 0.0 ? dx / rxy : 1.0, sp = rxy > 0.0 ? dy / rxy : 0.0;
        double rl = 1.0;
        for (int q = 0; q < S.l; ++q) rl *= rr;
        for (int q = 0; q < ncomp; ++q) {
            const int m = molden_m(S.l, q), am = m < 0 ? -m : m;
            double cm = 1.0, sm = 0.0;                   // cos(am phi), sin(am phi)
            for (int t = 0; t < am; ++t) {
                const double cn = cm * cp - sm * sp;
                sm = sm * cp + cm * sp;
                cm = cn;
            }
            const double sl = s_lm(S.l, am, c, s);
            const double y = m == 0 ? sl : 1.41421356237309504880 * sl * (m > 0 ? cm : sm);
            out[q] = rl * y * rad;
        }
    }
}

// rho[p] = sum_i occ_i Psi[p + i Pc]^2 into column n_mo of Psi; with
// vx_coef != 0 the local exchange potential -vx_coef rho^(1/3)
// (LocalExchange.hpp: (3/pi)^(1/3) for Slater, 1.5 (3/pi)^(1/3) for
// Kohn-Sham) into column n_mo + 1
__global__ void k_density(double* __restrict__ Psi, const double* __restrict__ occ, int n_mo, long Pc,
                          double vx_coef) {
    for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < Pc; p += (long)gridDim.x * blockDim.x) {
        double rho = 0.0;
        for (int i = 0; i < n_mo; ++i) {
            const double v = Psi[p + (size_t)i * Pc];
            rho += occ[i] * v * v;
        }
        Psi[p + (size_t)n_mo * Pc] = rho;
        if (vx_coef != 0.0) Psi[p + (size_t)(n_mo + 1) * Pc] = -vx_coef * cbrt(fmax(0.0, rho));
    }
}

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
    const int nT = Lmax + 1, nP = 2 * (Lmax + 1), nM = 2 * Lmax + 1;
    const long n_lm = (long)(Lmax + 1) * (Lmax + 1);
    // radial points per device pass: samples, C1, Q and the gathered rows within 64 Mi doubles
    const long per_pt = (long)nT * nP + (long)nT * nM + 2 * n_lm;
    int R = chunk > 0 ? chunk : (int)std::max<long>(1, (64L << 20) / per_pt);
    R = std::min(R, Nr);
    if ((long)R * nT > (1L << 30)) R = (int)std::max<long>(1, (1L << 30) / nT);
    SceStream st;
    SCATT_CUDA_TRY(cudaStreamCreateWithFlags(&st.s, cudaStreamNonBlocking));
    const cudaStream_t s = st.s;
    DevBuf<double> dX, dOut;
    SceProjector pj;
    SCATT_TRY(dX.alloc((size_t)R * nT * nP));
    SCATT_TRY(dOut.alloc((size_t)n_lm * R));
    SCATT_TRY(pj.init(Lmax, 1, R, s));
    for (int c0 = 0; c0 < Nr; c0 += R) {
        const int Rc = std::min(R, Nr - c0);
        SCATT_CUDA_TRY(cudaMemcpyAsync(dX.p, samples + (size_t)c0 * nT * nP, (size_t)Rc * nT * nP * sizeof(double),
                                       cudaMemcpyHostToDevice, s));
        SCATT_TRY(pj.run(dX.p, 0, Rc, dOut.p, s));
        SCATT_CUDA_TRY(cudaMemcpy2DAsync(F_lm + c0, (size_t)Nr * sizeof(double), dOut.p, (size_t)Rc * sizeof(double),
                                         (size_t)Rc * sizeof(double), (size_t)n_lm, cudaMemcpyDeviceToHost, s));
        SCATT_CUDA_TRY(cudaStreamSynchronize(s));        // the projector's entry tables are reused
    }
    return SCATT_OK;
}

int scatt_sce_basis(int Lmax, int Nr, double r0, double dr, const double* origin, int n_shell, const int* shell_l,
                    const int* shell_nprim, const double* shell_center, const double* exps, const double* coefs,
                    int n_mo, const double* C, const double* occ, int vx_form, int chunk, double* orb_lm,
                    double* rho_lm, double* vx_lm) {
    if (Lmax < 0 || Nr < 1 || !(dr > 0.0) || !origin || n_shell < 1 || !shell_l || !shell_nprim || !shell_center ||
        !exps || !coefs || n_mo < 1 || !C || !occ || vx_form < 0 || vx_form > 2 || (vx_form > 0) != (vx_lm != nullptr) ||
        (!orb_lm && !rho_lm && !vx_lm)) {
        set_last_error("scatt_sce_basis: need Lmax >= 0, Nr >= 1, dr > 0, shells, orbitals, vx_form 0 / 1 / 2 "
                       "with vx_lm given exactly when it is not 0, and an output");
        return SCATT_ERR_ARG;
    }
    // the normalised contraction of every shell (MoldenBasis.hpp:129-190, SphericalGaussian.hpp)
    std::vector<ShellDev> sh(n_shell);
    std::vector<double> ex, ct;
    int nbf = 0;
    for (int i = 0; i < n_shell; ++i) {
        const int l = shell_l[i], np = shell_nprim[i];
        if (l < 0 || l > 20 || np < 1) {
            set_last_error("scatt_sce_basis: shell " + std::to_string(i) + " needs 0 <= l <= 20 and primitives");
            return SCATT_ERR_ARG;
        }
        const double* e = exps + ex.size();
        const double* c = coefs + ex.size();
        double so = 0.0;
        for (int a = 0; a < np; ++a)
            for (int b = 0; b < np; ++b)
                so += c[a] * c[b] * std::pow(2.0 * std::sqrt(e[a] * e[b]) / (e[a] + e[b]), l + 1.5);
        if (!(so > 0.0)) {
            set_last_error("build_basis: non-positive self-overlap");
            return SCATT_ERR_ARG;
        }
        double dfact = 1.0;
        for (int k = 1; k <= l; ++k) dfact *= 2.0 * k + 1.0;
        sh[i] = ShellDev{shell_center[3 * i], shell_center[3 * i + 1], shell_center[3 * i + 2], l, np, (int)ex.size(),
                         nbf};
        for (int a = 0; a < np; ++a) {
            const double nsph = std::sqrt(std::pow(2.0, 2.0 * l + 3.5) * std::pow(e[a], l + 1.5) /
                                          (std::sqrt(SCE_PI) * dfact));
            ex.push_back(e[a]);
            ct.push_back(c[a] / std::sqrt(so) * nsph);
        }
        nbf += l == 0 ? 1 : 2 * l + 1;
    }
    SCATT_TRY(require_device());
    const int nT = Lmax + 1, nP = 2 * (Lmax + 1), nM = 2 * Lmax + 1, n_fn = n_mo + (vx_form ? 2 : 1);
    const long n_lm = (long)(Lmax + 1) * (Lmax + 1), nTP = (long)nT * nP;
    const double cbrt3pi = std::cbrt(3.0 / SCE_PI);
    const double vx_coef = vx_form == 1 ? cbrt3pi : vx_form == 2 ? 1.5 * cbrt3pi : 0.0;
    const long per_pt = nTP * (nbf + n_fn) + (long)n_fn * (nT * nM + 2 * n_lm);
    int R = chunk > 0 ? chunk : (int)std::max<long>(1, (64L << 20) / per_pt);
    R = std::min(R, Nr);
    if ((long)R * nTP > (1L << 30)) R = (int)std::max<long>(1, (1L << 30) / nTP);
    SceStream st;
    SCATT_CUDA_TRY(cudaStreamCreateWithFlags(&st.s, cudaStreamNonBlocking));
    const cudaStream_t s = st.s;
    SceProjector pj;
    SCATT_TRY(pj.init(Lmax, n_fn, R, s));
    // unit directions of the grid, [theta][phi]
    std::vector<double> dirh(3 * nTP);
    for (int i = 0; i < nT; ++i) {
        const double st_ = std::sqrt(std::max(0.0, 1.0 - pj.x[i] * pj.x[i]));
        for (int j = 0; j < nP; ++j) {
            const double ph = 2.0 * SCE_PI * j / nP;
            double* d = dirh.data() + 3 * ((long)i * nP + j);
            d[0] = st_ * std::cos(ph);
            d[1] = st_ * std::sin(ph);
            d[2] = pj.x[i];
        }
    }
    DevBuf<ShellDev> dsh;
    DevBuf<double> dex, dct, ddir, dC, docc, dPhi, dPsi, dOut;
    SCATT_TRY(dsh.upload(sh, s));
    SCATT_TRY(dex.upload(ex, s));
    SCATT_TRY(dct.upload(ct, s));
    SCATT_TRY(ddir.upload(dirh, s));
    SCATT_TRY(dC.upload(C, (size_t)n_mo * nbf, s));
    SCATT_TRY(docc.upload(occ, (size_t)n_mo, s));
    SCATT_TRY(dPhi.alloc((size_t)R * nTP * nbf));
    SCATT_TRY(dPsi.alloc((size_t)R * nTP * n_fn));
    SCATT_TRY(dOut.alloc((size_t)n_fn * n_lm * R));
    DevBuf<GemmEntry> dent;
    SCATT_TRY(dent.alloc(1));
    for (int c0 = 0; c0 < Nr; c0 += R) {
        const int Rc = std::min(R, Nr - c0);
        const long Pc = (long)Rc * nTP;
        const long tot = Pc * n_shell;
        k_ao_eval<<<(int)std::max<long>(1, std::min<long>((tot + 255) / 256, 148L * 16)), 256, 0, s>>>(
            dsh.p, n_shell, dex.p, dct.p, ddir.p, (int)nTP, (int)Pc, origin[0], origin[1], origin[2], r0, dr, c0, nbf,
            dPhi.p);
        SCATT_COUNT_LAUNCH(1);
        // Psi^T (Pc x n_mo) = Phi^T C^T: the orbitals' samples, one contiguous column each
        const GemmEntry e{dPhi.p, dC.p, dPsi.p, (int)Pc, n_mo, nbf, nbf, nbf, (int)Pc, 1.0, 0.0};
        SCATT_CUDA_TRY(cudaMemcpyAsync(dent.p, &e, sizeof(GemmEntry), cudaMemcpyHostToDevice, s));
        SCATT_TRY(gemm_batched(dent.p, 1, (int)Pc, n_mo, 1, 0, s));
        k_density<<<(int)std::max<long>(1, std::min<long>((Pc + 255) / 256, 148L * 8)), 256, 0, s>>>(dPsi.p, docc.p,
                                                                                                    n_mo, Pc, vx_coef);
        SCATT_COUNT_LAUNCH(1);
        SCATT_CUDA_TRY(cudaGetLastError());
        SCATT_TRY(pj.run(dPsi.p, Pc, Rc, dOut.p, s));
        for (int f = 0; f < n_fn; ++f) {
            double* dst = f < n_mo ? (orb_lm ? orb_lm + (size_t)f * n_lm * Nr : nullptr) : (f == n_mo ? rho_lm : vx_lm);
            if (!dst) continue;
            SCATT_CUDA_TRY(cudaMemcpy2DAsync(dst + c0, (size_t)Nr * sizeof(double), dOut.p + (size_t)f * n_lm * Rc,
                                             (size_t)Rc * sizeof(double), (size_t)Rc * sizeof(double), (size_t)n_lm,
                                             cudaMemcpyDeviceToHost, s));
        }
        SCATT_CUDA_TRY(cudaStreamSynchronize(s));        // the entry tables are reused
    }
    return SCATT_OK;
}

}  // extern "C"
