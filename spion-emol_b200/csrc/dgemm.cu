// dgemm.cu -- batched FP64 GEMM on the sm_100a FP64 tensor-core path.
//
// Three kernels by the batch's largest M: thin (M <= 16, 16 x 64 tiles),
// general (64 x 64 tiles) and pipelined (M >= 128, 128 x 64 tiles fed by a
// cp.async ring).  In the general kernel each CTA computes a 64 x 64 tile of
// C for one batch entry with four warps (2 x 2, 32 x 32 per warp) issuing
// mma.sync.m16n8k4 f64 (DMMA) from double-buffered shared-memory tiles of
// depth 16.  Operands are staged through registers so the next K-tile's
// global loads overlap the current tile's tensor-core work.  Transposes are
// resolved at load time (opA, opB template flags), so A^T B, A B^T, ... need
// no extra pass.
//
// Entries flagged sym (a symmetric product added to a symmetric C) compute
// only the lower-triangle tiles and mirror each result.
//
// This is the contraction engine behind the Schur complement
// S = A - (B D^-1) B^T, the W^-1 blocks (Sinv B, B^T Sinv B), the dipole /
// overlap row sweeps and the outer-region products.
#include "common.cuh"

#include <atomic>
#include <cstdint>

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

// Large products (some entry M >= 128: the Schur update B D^-1 B^T, T =
// Sinv Bs, F = Bs^T T, the fit rows): 128 x 64 tiles, eight warps of
// 32 x 32, two CTAs per SM.  k streams through a two-stage cp.async ring of
// 32-deep stages, so a stage lands while the previous one is multiplied.
// Each operand is staged in the layout its global storage is contiguous in
// (A as [k][m] for op N, [m][k] for op T; B as [n][k] for op N, [k][n] for
// op T), so every copy is a contiguous run: 16-byte copies where the leading
// dimension, the contiguous extent and the base allow, 8-byte otherwise.
// Row strides are 4 mod 16 doubles, which keeps the fragment reads free of
// bank conflicts in every layout.
constexpr int PBM = 128, PBN = 64, PBK = 32, PTHREADS = 256;
constexpr int PA_MK = PBM + 4;               // [k][m] rows
constexpr int PA_KM = PBK + 4;               // [m][k] rows
constexpr int PB_NK = PBK + 4;               // [n][k] rows
constexpr int PB_KN = PBN + 4;               // [k][n] rows

template <int OPA, int OPB>
struct PipeLayout {
    static constexpr int A_ELEMS = OPA == 0 ? PBK * PA_MK : PBM * PA_KM;
    static constexpr int B_ELEMS = OPB == 0 ? PBN * PB_NK : PBK * PB_KN;
    static constexpr int STAGE = A_ELEMS + B_ELEMS;
    static constexpr size_t SMEM = 2 * (size_t)STAGE * sizeof(double);
};

__device__ __forceinline__ void pipe_cp8(double* sdst, const double* gsrc, bool pred) {
    const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(sdst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" :: "r"(sa), "l"(gsrc), "r"(pred ? 8 : 0));
}
__device__ __forceinline__ void pipe_cp16(double* sdst, const double* gsrc, bool pred) {
    const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(sdst));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" :: "r"(sa), "l"(gsrc), "r"(pred ? 16 : 0));
}

template <int OPA, int OPB>
__global__ void __launch_bounds__(PTHREADS, 2)
gemm_pipe_kernel(const GemmEntry* __restrict__ entries) {
    using L = PipeLayout<OPA, OPB>;
    const GemmEntry e = entries[blockIdx.z];
    const int m0 = blockIdx.x * PBM;
    const int n0 = blockIdx.y * PBN;
    if (m0 >= e.M || n0 >= e.N) return;
    const bool sym = e.sym != 0;
    if (sym && n0 > m0 + PBM - 1) return;        // strictly upper tiles come from the mirror

    extern __shared__ double psmem[];
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int wm = (warp & 3) * 32, wn = (warp >> 2) * 32;
    // 16-byte copies: even leading dimension, even contiguous extent, 16-byte aligned base
    const bool a16 = (e.lda % 2 == 0) && ((OPA == 0 ? e.M : e.K) % 2 == 0) &&
                     ((reinterpret_cast<uintptr_t>(e.A) & 15) == 0);
    const bool b16 = (e.ldb % 2 == 0) && ((OPB == 0 ? e.K : e.N) % 2 == 0) &&
                     ((reinterpret_cast<uintptr_t>(e.B) & 15) == 0);
    const int nk = (e.K + PBK - 1) / PBK;

    auto issue = [&](int kt) {
        double* As = psmem + (size_t)(kt & 1) * L::STAGE;
        double* Bs = As + L::A_ELEMS;
        const int k0 = kt * PBK;
        if (OPA == 0) {                           // A(m, k) = A[m + k lda]: [k][m]
            if (a16) {
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const int idx = tid + u * PTHREADS;
                    const int k = idx >> 6, m = 2 * (idx & 63);
                    const bool ok = m0 + m < e.M && k0 + k < e.K;
                    pipe_cp16(As + k * PA_MK + m, e.A + (ok ? (m0 + m) + (size_t)(k0 + k) * e.lda : 0), ok);
                }
            } else {
#pragma unroll 4
                for (int u = 0; u < 16; ++u) {
                    const int idx = tid + u * PTHREADS;
                    const int k = idx >> 7, m = idx & 127;
                    const bool ok = m0 + m < e.M && k0 + k < e.K;
                    pipe_cp8(As + k * PA_MK + m, e.A + (ok ? (m0 + m) + (size_t)(k0 + k) * e.lda : 0), ok);
                }
            }
        } else {                                  // A(m, k) = A[k + m lda]: [m][k]
            if (a16) {
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const int idx = tid + u * PTHREADS;
                    const int m = idx >> 4, k = 2 * (idx & 15);
                    const bool ok = m0 + m < e.M && k0 + k < e.K;
                    pipe_cp16(As + m * PA_KM + k, e.A + (ok ? (k0 + k) + (size_t)(m0 + m) * e.lda : 0), ok);
                }
            } else {
#pragma unroll 4
                for (int u = 0; u < 16; ++u) {
                    const int idx = tid + u * PTHREADS;
                    const int m = idx >> 5, k = idx & 31;
                    const bool ok = m0 + m < e.M && k0 + k < e.K;
                    pipe_cp8(As + m * PA_KM + k, e.A + (ok ? (k0 + k) + (size_t)(m0 + m) * e.lda : 0), ok);
                }
            }
        }
        if (OPB == 0) {                           // B(k, n) = B[k + n ldb]: [n][k]
            if (b16) {
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int idx = tid + u * PTHREADS;
                    const int n = idx >> 4, k = 2 * (idx & 15);
                    const bool ok = n0 + n < e.N && k0 + k < e.K;
                    pipe_cp16(Bs + n * PB_NK + k, e.B + (ok ? (k0 + k) + (size_t)(n0 + n) * e.ldb : 0), ok);
                }
            } else {
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const int idx = tid + u * PTHREADS;
                    const int n = idx >> 5, k = idx & 31;
                    const bool ok = n0 + n < e.N && k0 + k < e.K;
                    pipe_cp8(Bs + n * PB_NK + k, e.B + (ok ? (k0 + k) + (size_t)(n0 + n) * e.ldb : 0), ok);
                }
            }
        } else {                                  // B(k, n) = B[n + k ldb]: [k][n]
            if (b16) {
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int idx = tid + u * PTHREADS;
                    const int k = idx >> 5, n = 2 * (idx & 31);
                    const bool ok = n0 + n < e.N && k0 + k < e.K;
                    pipe_cp16(Bs + k * PB_KN + n, e.B + (ok ? (n0 + n) + (size_t)(k0 + k) * e.ldb : 0), ok);
                }
            } else {
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const int idx = tid + u * PTHREADS;
                    const int k = idx >> 6, n = idx & 63;
                    const bool ok = n0 + n < e.N && k0 + k < e.K;
                    pipe_cp8(Bs + k * PB_KN + n, e.B + (ok ? (n0 + n) + (size_t)(k0 + k) * e.ldb : 0), ok);
                }
            }
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    };

    double acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int v = 0; v < 4; ++v) acc[i][j][v] = 0.0;

    if (nk > 0) issue(0);
    if (nk > 1) issue(1);
#pragma unroll 1
    for (int kt = 0; kt < nk; ++kt) {
        if (kt + 1 < nk) asm volatile("cp.async.wait_group 1;\n" ::: "memory");
        else asm volatile("cp.async.wait_group 0;\n" ::: "memory");
        __syncthreads();
        const double* As = psmem + (size_t)(kt & 1) * L::STAGE;
        const double* Bs = As + L::A_ELEMS;
#pragma unroll
        for (int kk = 0; kk < PBK; kk += 4) {
            double a[2][2], b[4];
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const int r = wm + i * 16 + g;
                if (OPA == 0) {
                    a[i][0] = As[(kk + t) * PA_MK + r];
                    a[i][1] = As[(kk + t) * PA_MK + r + 8];
                } else {
                    a[i][0] = As[r * PA_KM + kk + t];
                    a[i][1] = As[(r + 8) * PA_KM + kk + t];
                }
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int c = wn + j * 8 + g;
                b[j] = (OPB == 0) ? Bs[c * PB_NK + kk + t] : Bs[(kk + t) * PB_KN + c];
            }
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) dmma_16x8x4(acc[i][j], a[i][0], a[i][1], b[j]);
        }
        if (kt + 2 < nk) {
            __syncthreads();                     // every warp is done with this stage
            issue(kt + 2);
        }
    }

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

template <int OPA, int OPB>
int launch_pipe(const GemmEntry* entries_dev, int count, int maxM, int maxN, cudaStream_t stream) {
    using L = PipeLayout<OPA, OPB>;
    static_assert(L::SMEM <= 113 * 1024, "two CTAs per SM");
    int dev = 0;
    SCATT_CUDA_TRY(cudaGetDevice(&dev));
    static std::atomic<unsigned long long> done{0};
    if (dev >= 0 && dev < 64 && !(done.load() & (1ull << dev))) {
        SCATT_CUDA_TRY(cudaFuncSetAttribute(gemm_pipe_kernel<OPA, OPB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)L::SMEM));
        done.fetch_or(1ull << dev);
    }
    const dim3 grid((maxM + PBM - 1) / PBM, (maxN + PBN - 1) / PBN, count);
    gemm_pipe_kernel<OPA, OPB><<<grid, PTHREADS, L::SMEM, stream>>>(entries_dev);
    return SCATT_OK;
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
    if (maxM >= PBM) {
        if (opA == 0 && opB == 0)      SCATT_TRY((launch_pipe<0, 0>(entries_dev, count, maxM, maxN, stream)));
        else if (opA == 1 && opB == 0) SCATT_TRY((launch_pipe<1, 0>(entries_dev, count, maxM, maxN, stream)));
        else if (opA == 0 && opB == 1) SCATT_TRY((launch_pipe<0, 1>(entries_dev, count, maxM, maxN, stream)));
        else                           SCATT_TRY((launch_pipe<1, 1>(entries_dev, count, maxM, maxN, stream)));
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
