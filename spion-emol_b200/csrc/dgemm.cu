// dgemm.cu -- batched FP64 GEMM on the sm_100a FP64 tensor-core path.
//
// Each CTA computes a 64 x 64 tile of C for one batch entry with four warps
// (2 x 2, 32 x 32 per warp) issuing mma.sync.m16n8k4 f64 (DMMA) from
// double-buffered shared-memory tiles of depth 16.  Operands are staged
// through registers so the next K-tile's global loads overlap the current
// tile's tensor-core work.  Transposes are resolved at load time (opA, opB
// template flags), so A^T B, A B^T, ... need no extra pass.
//
// Entries flagged sym (a symmetric product added to a symmetric C) compute
// only the lower-triangle tiles and mirror each result.
//
// This is the contraction engine behind the Schur complement
// S = A - (B D^-1) B^T, the W^-1 blocks (Sinv B, B^T Sinv B), the dipole /
// overlap row sweeps and the outer-region products.
#include "common.cuh"

namespace scatt {

namespace {

constexpr int BM = 64, BN = 64, BK = 16, PAD = 4;
constexpr int THREADS = 128;

__device__ __forceinline__ void dmma_16x8x4(double (&c)[4], double a0, double a1, double b0) {
    asm volatile(
        "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 "
        "{%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
        : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
        : "d"(a0), "d"(a1), "d"(b0));
}

template <int OPA, int OPB>
__global__ void __launch_bounds__(THREADS)
gemm_kernel(const GemmEntry* __restrict__ entries) {
    const GemmEntry e = entries[blockIdx.z];
    const int m0 = blockIdx.x * BM;
    const int n0 = blockIdx.y * BN;
    if (m0 >= e.M || n0 >= e.N) return;
    const bool sym = e.sym != 0;
    if (sym && n0 > m0) return;                 // strictly upper tiles come from the mirror

    __shared__ double As[2][BK][BM + PAD];
    __shared__ double Bs[2][BK][BN + PAD];

    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int wm = (warp & 1) * 32, wn = (warp >> 1) * 32;

    double acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int v = 0; v < 4; ++v) acc[i][j][v] = 0.0;

    double ra[8], rb[8];
    const int nk = (e.K + BK - 1) / BK;

    auto load_tile = [&](int kt) {
        const int k0 = kt * BK;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            int m, k;
            if (OPA == 0) { m = tid & 63; k = (tid >> 6) + 2 * i; }
            else          { k = tid & 15; m = (tid >> 4) + 8 * i; }
            const int gm = m0 + m, gk = k0 + k;
            double v = 0.0;
            if (gm < e.M && gk < e.K)
                v = (OPA == 0) ? e.A[gm + (size_t)gk * e.lda] : e.A[gk + (size_t)gm * e.lda];
            ra[i] = v;
        }
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            int n, k;
            if (OPB == 0) { k = tid & 15; n = (tid >> 4) + 8 * i; }
            else          { n = tid & 63; k = (tid >> 6) + 2 * i; }
            const int gn = n0 + n, gk = k0 + k;
            double v = 0.0;
            if (gn < e.N && gk < e.K)
                v = (OPB == 0) ? e.B[gk + (size_t)gn * e.ldb] : e.B[gn + (size_t)gk * e.ldb];
            rb[i] = v;
        }
    };
    auto store_tile = [&](int buf) {
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            int m, k;
            if (OPA == 0) { m = tid & 63; k = (tid >> 6) + 2 * i; }
            else          { k = tid & 15; m = (tid >> 4) + 8 * i; }
            As[buf][k][m] = ra[i];
        }
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            int n, k;
            if (OPB == 0) { k = tid & 15; n = (tid >> 4) + 8 * i; }
            else          { n = tid & 63; k = (tid >> 6) + 2 * i; }
            Bs[buf][k][n] = rb[i];
        }
    };

    if (nk > 0) {
        load_tile(0);
        store_tile(0);
    }
    __syncthreads();

    for (int kt = 0; kt < nk; ++kt) {
        const int buf = kt & 1;
        if (kt + 1 < nk) load_tile(kt + 1);
#pragma unroll
        for (int kk = 0; kk < BK; kk += 4) {
            double a[2][2], b[4];
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                a[i][0] = As[buf][kk + t][wm + i * 16 + g];
                a[i][1] = As[buf][kk + t][wm + i * 16 + g + 8];
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[buf][kk + t][wn + j * 8 + g];
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) dmma_16x8x4(acc[i][j], a[i][0], a[i][1], b[j]);
        }
        if (kt + 1 < nk) store_tile(buf ^ 1);
        __syncthreads();
    }

    // Epilogue: C = alpha * acc + beta * C.
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                const int row = m0 + wm + i * 16 + g + ((v >> 1) << 3);
                const int col = n0 + wn + j * 8 + 2 * t + (v & 1);
                if (row < e.M && col < e.N && !(sym && col > row)) {
                    double* c = e.C + row + (size_t)col * e.ldc;
                    double r = e.alpha * acc[i][j][v];
                    if (e.beta != 0.0) r += e.beta * *c;
                    *c = r;
                    if (sym && col != row) e.C[col + (size_t)row * e.ldc] = r;
                }
            }
}

// Thin products (every entry M <= 16: the dipole / overlap row sweeps
// G(n) = G(n-1) Rinv(n) and their W^-1 terms, K_rows x N_t x N_t).  A
// 64-row tile would spend three quarters of its DMMAs on zero rows and make
// these HBM-bound sweeps compute-bound; here a CTA computes 16 x 64 of C
// with four warps of 16 x 16 and streams op(B) in 32-deep k tiles, staged
// through registers and double-buffered in shared memory as above.
constexpr int TBM = 16, TBN = 64, TBK = 32;

template <int OPA, int OPB>
__global__ void __launch_bounds__(THREADS)
gemm_thin_kernel(const GemmEntry* __restrict__ entries) {
    const GemmEntry e = entries[blockIdx.z];
    const int n0 = blockIdx.y * TBN;
    if (e.M <= 0 || n0 >= e.N) return;
    const bool sym = e.sym != 0;
    if (sym && n0 > 0) return;                  // M = N <= 16: one tile holds the lower triangle

    __shared__ double As[2][TBK][TBM + PAD];
    __shared__ double Bs[2][TBK][TBN + PAD];

    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int wn = warp * 16;

    double acc[2][4];
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int v = 0; v < 4; ++v) acc[j][v] = 0.0;

    double ra[4], rb[16];
    const int nk = (e.K + TBK - 1) / TBK;

    auto a_at = [&](int i, int& m, int& k) {
        if (OPA == 0) { m = tid & 15; k = (tid >> 4) + 8 * i; }
        else          { k = tid & 31; m = (tid >> 5) + 4 * i; }
    };
    auto b_at = [&](int i, int& n, int& k) {
        if (OPB == 0) { k = tid & 31; n = (tid >> 5) + 4 * i; }
        else          { n = tid & 63; k = (tid >> 6) + 2 * i; }
    };
    auto load_tile = [&](int kt) {
        const int k0 = kt * TBK;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            int m, k;
            a_at(i, m, k);
            const int gk = k0 + k;
            double v = 0.0;
            if (m < e.M && gk < e.K)
                v = (OPA == 0) ? e.A[m + (size_t)gk * e.lda] : e.A[gk + (size_t)m * e.lda];
            ra[i] = v;
        }
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            int n, k;
            b_at(i, n, k);
            const int gn = n0 + n, gk = k0 + k;
            double v = 0.0;
            if (gn < e.N && gk < e.K)
                v = (OPB == 0) ? e.B[gk + (size_t)gn * e.ldb] : e.B[gn + (size_t)gk * e.ldb];
            rb[i] = v;
        }
    };
    auto store_tile = [&](int buf) {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            int m, k;
            a_at(i, m, k);
            As[buf][k][m] = ra[i];
        }
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            int n, k;
            b_at(i, n, k);
            Bs[buf][k][n] = rb[i];
        }
    };

    if (nk > 0) {
        load_tile(0);
        store_tile(0);
    }
    __syncthreads();

    for (int kt = 0; kt < nk; ++kt) {
        const int buf = kt & 1;
        if (kt + 1 < nk) load_tile(kt + 1);
#pragma unroll
        for (int kk = 0; kk < TBK; kk += 4) {
            const double a0 = As[buf][kk + t][g];
            const double a1 = As[buf][kk + t][g + 8];
#pragma unroll
            for (int j = 0; j < 2; ++j) dmma_16x8x4(acc[j], a0, a1, Bs[buf][kk + t][wn + j * 8 + g]);
        }
        if (kt + 1 < nk) store_tile(buf ^ 1);
        __syncthreads();
    }

#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const int row = g + ((v >> 1) << 3);
            const int col = n0 + wn + j * 8 + 2 * t + (v & 1);
            if (row < e.M && col < e.N && !(sym && col > row)) {
                double* c = e.C + row + (size_t)col * e.ldc;
                double r = e.alpha * acc[j][v];
                if (e.beta != 0.0) r += e.beta * *c;
                *c = r;
                if (sym && col != row) e.C[col + (size_t)row * e.ldc] = r;
            }
        }
}

}  // namespace

int gemm_batched(const GemmEntry* entries_dev, int count, int maxM, int maxN,
                 int opA, int opB, cudaStream_t stream) {
    if (count <= 0 || maxM <= 0 || maxN <= 0) return SCATT_OK;
    if (count > 65535) {
        set_last_error("gemm_batched: batch count exceeds 65535");
        return SCATT_ERR_ARG;
    }
    if (maxM <= TBM) {
        const dim3 tg(1, (maxN + TBN - 1) / TBN, count);
        if (opA == 0 && opB == 0)      gemm_thin_kernel<0, 0><<<tg, THREADS, 0, stream>>>(entries_dev);
        else if (opA == 1 && opB == 0) gemm_thin_kernel<1, 0><<<tg, THREADS, 0, stream>>>(entries_dev);
        else if (opA == 0 && opB == 1) gemm_thin_kernel<0, 1><<<tg, THREADS, 0, stream>>>(entries_dev);
        else                           gemm_thin_kernel<1, 1><<<tg, THREADS, 0, stream>>>(entries_dev);
        SCATT_CUDA_TRY(cudaGetLastError());
        SCATT_COUNT_LAUNCH(1);
        return SCATT_OK;
    }
    dim3 grid((maxM + BM - 1) / BM, (maxN + BN - 1) / BN, count);
    if (opA == 0 && opB == 0)      gemm_kernel<0, 0><<<grid, THREADS, 0, stream>>>(entries_dev);
    else if (opA == 1 && opB == 0) gemm_kernel<1, 0><<<grid, THREADS, 0, stream>>>(entries_dev);
    else if (opA == 0 && opB == 1) gemm_kernel<0, 1><<<grid, THREADS, 0, stream>>>(entries_dev);
    else                           gemm_kernel<1, 1><<<grid, THREADS, 0, stream>>>(entries_dev);
    SCATT_CUDA_TRY(cudaGetLastError());
    SCATT_COUNT_LAUNCH(1);
    return SCATT_OK;
}

}  // namespace scatt
