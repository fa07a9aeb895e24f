// eig.cu -- eigenvalues of symmetric matrices on the device.
//
// Used for (a) the Johnson stability shift of SchurInverter
// (SchurInverter.cpp:44-59: smallest eigenvalue when the Gershgorin bound is
// inconclusive; the reference calls Eigen's SelfAdjointEigenSolver on the
// lower triangle) and (b) the eigenphases atan(eig K) of
// KMatrixExtractor.cpp:185-191 / AsymptoticAmplitudes.cpp:340-344.
//
// Method: Householder reduction to tridiagonal form (one CTA per matrix,
// reading only the lower triangle, in place in global memory), then
// Sturm-sequence bisection for the requested eigenvalues.  Both steps are
// backward stable, so eigenvalues are accurate to O(eps ||M||), the same
// guarantee the reference's QR-based solver gives.
#include <cmath>

#include "common.cuh"
#include "eig.cuh"

namespace scatt {

namespace {

constexpr int ET = 256;

__device__ double block_sum(double v, double* red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[w] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0) {
        for (int i = 0; i < ET / 32; ++i) s += red[i];
        red[ET / 32] = s;
    }
    __syncthreads();
    return red[ET / 32];
}

// Sturm count: number of eigenvalues of the tridiagonal (d, e) below x.
__device__ int sturm_count(const double* d, const double* e, int n, double x) {
    int cnt = 0;
    double q = d[0] - x;
    if (q < 0.0) ++cnt;
    for (int i = 1; i < n; ++i) {
        if (q == 0.0) q = 1e-300;
        q = (d[i] - x) - e[i - 1] * e[i - 1] / q;
        if (q < 0.0) ++cnt;
    }
    return cnt;
}

__device__ double bisect_kth(const double* d, const double* e, int n, int kth, double lo, double hi) {
    // smallest x with count(x) > kth
    for (int it = 0; it < 200; ++it) {
        const double mid = 0.5 * (lo + hi);
        if (mid <= lo || mid >= hi) break;
        if (sturm_count(d, e, n, mid) > kth) hi = mid; else lo = mid;
    }
    return 0.5 * (lo + hi);
}

__global__ void __launch_bounds__(ET)
tridiag_kernel(const EigEntry* __restrict__ entries) {
    const EigEntry en = entries[blockIdx.x];
    const int n = en.n;
    double* M = en.M;
    const int ld = en.ld;
    double* d = en.d;
    double* e = en.e;
    double* v = en.work;          // n
    double* p = en.work + n;      // n
    __shared__ double red[ET / 32 + 1];
    __shared__ double s_alpha, s_beta;
    const int tid = threadIdx.x;
    // only the lower triangle is read: mirror it into the upper triangle first
    for (int j = 0; j < n; ++j)
        for (int i = j + 1 + tid; i < n; i += ET) M[j + (size_t)i * ld] = M[i + (size_t)j * ld];
    __syncthreads();
    for (int k = 0; k + 2 < n; ++k) {
        // x = M[k+1:n, k]
        double ss = 0.0;
        for (int i = k + 1 + tid; i < n; i += ET) {
            const double x = M[i + (size_t)k * ld];
            ss += x * x;
        }
        const double nrm2 = block_sum(ss, red);
        if (tid == 0) {
            const double x0 = M[(k + 1) + (size_t)k * ld];
            const double nrm = sqrt(nrm2);
            double alpha = (x0 > 0.0) ? -nrm : nrm;
            double beta = 0.0;                      // 2 / (v^T v)
            if (nrm2 > 0.0) {
                const double vtv = nrm2 - x0 * x0 + (x0 - alpha) * (x0 - alpha);
                beta = vtv > 0.0 ? 2.0 / vtv : 0.0;
            } else {
                alpha = 0.0;
            }
            s_alpha = alpha;
            s_beta = beta;
            d[k] = M[k + (size_t)k * ld];
            e[k] = alpha;
        }
        __syncthreads();
        const double alpha = s_alpha, beta = s_beta;
        for (int i = k + 1 + tid; i < n; i += ET) {
            double x = M[i + (size_t)k * ld];
            if (i == k + 1) x -= alpha;
            v[i] = x;
        }
        __syncthreads();
        if (beta == 0.0) continue;
        // p = beta * A_sub v
        for (int i = k + 1 + tid; i < n; i += ET) {
            double s = 0.0;
            for (int j = k + 1; j < n; ++j) s += M[i + (size_t)j * ld] * v[j];
            p[i] = beta * s;
        }
        __syncthreads();
        // w = p - (beta/2) (p^T v) v
        double pv = 0.0;
        for (int i = k + 1 + tid; i < n; i += ET) pv += p[i] * v[i];
        const double K = 0.5 * beta * block_sum(pv, red);
        for (int i = k + 1 + tid; i < n; i += ET) p[i] -= K * v[i];
        __syncthreads();
        // A_sub -= v w^T + w v^T
        for (int j = k + 1; j < n; ++j) {
            const double vj = v[j], wj = p[j];
            for (int i = k + 1 + tid; i < n; i += ET)
                M[i + (size_t)j * ld] -= v[i] * wj + p[i] * vj;
        }
        __syncthreads();
    }
    if (tid == 0) {
        if (n >= 2) {
            d[n - 2] = M[(n - 2) + (size_t)(n - 2) * ld];
            e[n - 2] = M[(n - 1) + (size_t)(n - 2) * ld];
        }
        d[n - 1] = M[(n - 1) + (size_t)(n - 1) * ld];
    }
}

// eigenvalues by bisection: one thread per requested eigenvalue index
__global__ void bisect_kernel(const EigEntry* __restrict__ entries, int nwant) {
    const EigEntry en = entries[blockIdx.y];
    const int n = en.n;
    const int kth = blockIdx.x * blockDim.x + threadIdx.x;
    const int want = nwant > 0 ? min(nwant, n) : n;
    if (kth >= want) return;
    double lo = INFINITY, hi = -INFINITY;
    for (int i = 0; i < n; ++i) {
        const double r = (i > 0 ? fabs(en.e[i - 1]) : 0.0) + (i + 1 < n ? fabs(en.e[i]) : 0.0);
        lo = fmin(lo, en.d[i] - r);
        hi = fmax(hi, en.d[i] + r);
    }
    const double pad = 1e-12 * fmax(fabs(lo), fabs(hi)) + 1e-300;
    en.out[kth] = bisect_kth(en.d, en.e, n, kth, lo - pad, hi + pad);
}

}  // namespace

int sym_eigvals_batched(const EigEntry* entries_dev, int count, int nmax, int nwant,
                        cudaStream_t stream) {
    if (count <= 0) return SCATT_OK;
    tridiag_kernel<<<count, ET, 0, stream>>>(entries_dev);
    const int want = nwant > 0 ? nwant : nmax;
    dim3 g((want + 127) / 128, count);
    bisect_kernel<<<g, 128, 0, stream>>>(entries_dev, nwant);
    SCATT_CUDA_TRY(cudaGetLastError());
    SCATT_COUNT_LAUNCH(2);
    return SCATT_OK;
}

}  // namespace scatt
