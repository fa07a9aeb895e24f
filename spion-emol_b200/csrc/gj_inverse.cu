// gj_inverse.cu -- batched FP64 matrix inversion, blocked Gauss-Jordan with
// partial (row) pivoting, for the per-step dense inverses of the Numerov
// R-ratio recurrence (R = 12 W^-1 - 10 I - Rinv_prev, N_total x N_total),
// the Schur inverses Sinv(n) and the small per-energy solves.
//
// The reference inverts with LU + partial pivoting (dgetrf + dgetri, or
// Eigen partialPivLu) and symmetrises with 0.5 (M + M^T)
// (src/scatt/LapackInverse.hpp:53-92, ForwardRPropagator.cpp:357-358).
// Gauss-Jordan with the same pivot rule (largest |entry| among rows not yet
// pivoted, first index on ties) computes the same inverse to rounding and
// is a better fit for the GPU: every block step is one uniform rank-16
// update of the whole matrix instead of a shrinking trailing matrix.
//
// Block step kb (columns K = [k0, k0 + 16)):
//   panel  : one CTA per matrix loads the n x 16 panel into shared memory,
//            runs 16 pivoted GJ eliminations on it (pivot search by warp
//            shuffles + one block reduction per column) and writes the
//            transformed panel M, the row map sigma of this step and the
//            running row identity.
//   update : a DMMA tile kernel applies the deferred update to every other
//            column:  new[i, c] = (i in K ? 0 : old[sigma(i), c])
//                                  + sum_j M[i, j] * old[sigma(k0 + j), c].
//            It reads the previous buffer and writes the other one
//            (ping-pong), so the row interchanges need no separate pass
//            and no CTA ever reads a value another CTA is writing.
// finalize: out[:, j] = X[:, pi(j)] with pi the inverse of the composite
//            row permutation (LAPACK getri's column interchanges), and
//            optionally 0.5 (X + X^T) in the same pass.
#include "common.cuh"

#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <string>
#include <tuple>

namespace scatt {

namespace {

constexpr int NB = GJ_NB;
constexpr int PANEL_THREADS = 512;
constexpr int PANEL_WARPS = PANEL_THREADS / 32;
constexpr size_t PANEL_SMEM_LIMIT = 227 * 1024 - 1024;   // dynamic part; static scratch stays below 1 KB

size_t panel_smem_bytes(int nmax) {
    return (size_t)nmax * NB * sizeof(double) + 2 * (size_t)nmax * sizeof(int)
           + PANEL_WARPS * (sizeof(double) + sizeof(int)) + 64;
}

__device__ __forceinline__ double* buf_of(const GjEntry& e, int which) {
    return which == 0 ? e.A : e.W;
}

__device__ __forceinline__ void better(double& v, int& i, double v2, int i2) {
    // larger magnitude wins; ties go to the smaller row index
    if (v2 > v || (v2 == v && i2 >= 0 && (i < 0 || i2 < i))) { v = v2; i = i2; }
}

__global__ void __launch_bounds__(PANEL_THREADS)
gj_panel_kernel(const GjEntry* __restrict__ entries, int kb) {
    const GjEntry e = entries[blockIdx.x];
    const int n = e.n;
    const int k0 = kb * NB;
    if (k0 >= n) return;
    const int nb = min(NB, n - k0);
    const double* src = buf_of(e, kb & 1);
    double* dst = buf_of(e, (kb + 1) & 1);

    // panel held column-major in shared memory: P[j * n + i] (consecutive
    // rows -> consecutive banks, so row-parallel sweeps are conflict-free)
    extern __shared__ double smem[];
    double* P = smem;
    int* loc = reinterpret_cast<int*>(P + (size_t)n * NB);
    int* rid = loc + n;
    double* red_v = reinterpret_cast<double*>(rid + n);
    int* red_i = reinterpret_cast<int*>(red_v + PANEL_WARPS);
    __shared__ int s_piv;
    __shared__ int s_status;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    if (tid == 0) s_status = (kb == 0) ? 0 : e.status[0];
    for (int j = 0; j < nb; ++j)
        for (int i = tid; i < n; i += PANEL_THREADS)
            P[j * n + i] = src[i + (size_t)(k0 + j) * e.ld];
    for (int i = tid; i < n; i += PANEL_THREADS) {
        loc[i] = i;
        rid[i] = (kb == 0) ? i : e.rowid[i];
    }
    __syncthreads();

    for (int j = 0; j < nb; ++j) {
        const int k = k0 + j;
        const double* Pj = P + j * n;
        // ---- pivot search over rows [k, n): largest |P|, first index on ties
        double bv = -1.0;
        int bi = -1;
        for (int i = k + tid; i < n; i += PANEL_THREADS) {
            const double v = fabs(Pj[i]);
            if (v > bv) { bv = v; bi = i; }
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            const double ov = __shfl_down_sync(0xffffffffu, bv, off);
            const int oi = __shfl_down_sync(0xffffffffu, bi, off);
            better(bv, bi, ov, oi);
        }
        if (lane == 0) { red_v[warp] = bv; red_i[warp] = bi; }
        __syncthreads();
        if (warp == 0) {
            bv = lane < PANEL_WARPS ? red_v[lane] : -1.0;
            bi = lane < PANEL_WARPS ? red_i[lane] : -1;
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                const double ov = __shfl_down_sync(0xffffffffu, bv, off);
                const int oi = __shfl_down_sync(0xffffffffu, bi, off);
                better(bv, bi, ov, oi);
            }
            if (lane == 0) {
                int p = bi;
                if (p < 0) {               // every candidate NaN
                    p = k;
                    if (s_status == 0) { s_status = DEV_NONFINITE; e.status[1] = k; }
                } else if (!(bv < INFINITY)) {
                    if (s_status == 0) { s_status = DEV_NONFINITE; e.status[1] = k; }
                } else if (bv == 0.0) {
                    if (s_status == 0) { s_status = DEV_SINGULAR; e.status[1] = k; }
                }
                s_piv = p;
            }
        }
        __syncthreads();
        const int p = s_piv;
        // ---- interchange rows k <-> p and scale the new pivot row (one phase)
        if (tid < nb) {
            double piv = P[j * n + p];
            if (piv == 0.0) piv = 1.0;             // status already records the failure
            const double inv = 1.0 / piv;
            const double a = P[tid * n + k];
            const double b = P[tid * n + p];
            P[tid * n + p] = a;
            P[tid * n + k] = (tid == j) ? inv : b * inv;
        } else if (tid == NB && p != k) {
            const int a = loc[k]; loc[k] = loc[p]; loc[p] = a;
            const int b = rid[k]; rid[k] = rid[p]; rid[p] = b;
        }
        __syncthreads();
        // ---- eliminate column j from every other row
        const double inv = P[j * n + k];
        for (int i = tid; i < n; i += PANEL_THREADS) {
            if (i == k) continue;
            const double f = P[j * n + i];
            if (f != 0.0) {
#pragma unroll
                for (int jj = 0; jj < NB; ++jj) {
                    if (jj < nb && jj != j) P[jj * n + i] -= f * P[jj * n + k];
                }
            }
            P[j * n + i] = -f * inv;
        }
        __syncthreads();
    }

    for (int j = 0; j < nb; ++j)
        for (int i = tid; i < n; i += PANEL_THREADS)
            dst[i + (size_t)(k0 + j) * e.ld] = P[j * n + i];
    for (int i = tid; i < n; i += PANEL_THREADS) {
        e.sigma[i] = loc[i];
        e.rowid[i] = rid[i];
    }
    if (tid == 0) e.status[0] = s_status;
}

// (|value|, index) key comparison: larger magnitude wins, ties go to the
// smaller index, NaN never wins.
__device__ __forceinline__ void better_key(double& v, int& i, double v2, int i2) {
    if (v2 > v || (v2 == v && i2 >= 0 && (i < 0 || i2 < i))) { v = v2; i = i2; }
}

// Single-level panel: W warps, R rows of 16 columns per thread in registers,
// with a rolled pivot loop: after each pivot the register window is
// rotated by one column, so the active column is always v[r][0] and every
// index stays static while the loop body stays small (instruction-cache
// resident).  Shared rows (scaled pivot row, old row k) are kept in the same
// rotated order; 16 rotations restore the original order.
template <int R, int MAXT>
__global__ void __launch_bounds__(MAXT, 1)
gj_panel5_kernel(const GjEntry* __restrict__ entries, int kb) {
    const GjEntry e = entries[blockIdx.x];
    const int n = e.n;
    const int k0 = kb * NB;
    if (k0 >= n) return;
    const int nb = min(NB, n - k0);
    const double* src = buf_of(e, kb & 1);
    double* dst = buf_of(e, (kb + 1) & 1);
    const int T = blockDim.x, W = T >> 5;

    extern __shared__ double smem[];
    int* loc = reinterpret_cast<int*>(smem);
    int* rid = loc + n;
    __shared__ double red_v[2][32];
    __shared__ int red_i[2][32];
    __shared__ double sprow[2][NB];
    __shared__ double krow[2][NB];
    __shared__ int s_status;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    double v[R][NB];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int i = tid + r * T;
#pragma unroll
        for (int j = 0; j < NB; ++j)
            v[r][j] = (i < n && j < nb) ? src[i + (size_t)(k0 + j) * e.ld] : 0.0;
    }
    for (int i = tid; i < n; i += T) {
        loc[i] = i;
        rid[i] = (kb == 0) ? i : e.rowid[i];
    }
    if (tid == 0) s_status = (kb == 0) ? 0 : e.status[0];
    __syncthreads();

#pragma unroll 1
    for (int j = 0; j < NB; ++j) {
        if (j < nb) {
            const int k = k0 + j;
            const int par = j & 1;
            double bv = -1.0;
            int bi = -1;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int i = tid + r * T;
                if (i >= k && i < n) {
                    const double a = fabs(v[r][0]);
                    if (a > bv) { bv = a; bi = i; }
                }
            }
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                const double ov = __shfl_xor_sync(0xffffffffu, bv, off);
                const int oi = __shfl_xor_sync(0xffffffffu, bi, off);
                better_key(bv, bi, ov, oi);
            }
            if (lane == 0) { red_v[par][warp] = bv; red_i[par][warp] = bi; }
            __syncthreads();
            bv = (lane < W) ? red_v[par][lane] : -1.0;
            bi = (lane < W) ? red_i[par][lane] : -1;
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                const double ov = __shfl_xor_sync(0xffffffffu, bv, off);
                const int oi = __shfl_xor_sync(0xffffffffu, bi, off);
                better_key(bv, bi, ov, oi);
            }
            const int p = bi < 0 ? k : bi;
            if (tid == 0) {
                int st = 0;
                if (bi < 0 || !(bv < INFINITY)) st = DEV_NONFINITE;
                else if (bv == 0.0) st = DEV_SINGULAR;
                if (st && s_status == 0) { s_status = st; e.status[1] = k; }
                if (p != k) {
                    const int a = loc[k]; loc[k] = loc[p]; loc[p] = a;
                    const int b2 = rid[k]; rid[k] = rid[p]; rid[p] = b2;
                }
            }
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int i = tid + r * T;
                if (i == p) {
                    double piv = v[r][0];
                    if (piv == 0.0) piv = 1.0;      // the status word records the failure
                    const double inv = 1.0 / piv;
                    sprow[par][0] = inv;
#pragma unroll
                    for (int c = 1; c < NB; ++c) sprow[par][c] = v[r][c] * inv;
                }
                if (i == k) {
#pragma unroll
                    for (int c = 0; c < NB; ++c) krow[par][c] = v[r][c];
                }
            }
            __syncthreads();
            const double inv = sprow[par][0];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int i = tid + r * T;
                if (i < n) {
                    if (i == k) {
#pragma unroll
                        for (int c = 0; c < NB; ++c) v[r][c] = sprow[par][c];
                    } else {
                        if (i == p) {
#pragma unroll
                            for (int c = 0; c < NB; ++c) v[r][c] = krow[par][c];
                        }
                        const double f = v[r][0];
                        v[r][0] = -f * inv;
#pragma unroll
                        for (int c = 1; c < NB; ++c) v[r][c] -= f * sprow[par][c];
                    }
                }
            }
        }
        // rotate the window: column j moves to the back, column j + 1 to the front
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const double t0 = v[r][0];
#pragma unroll
            for (int c = 0; c < NB - 1; ++c) v[r][c] = v[r][c + 1];
            v[r][NB - 1] = t0;
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int i = tid + r * T;
        if (i < n) {
#pragma unroll
            for (int j = 0; j < NB; ++j)
                if (j < nb) dst[i + (size_t)(k0 + j) * e.ld] = v[r][j];
        }
    }
    for (int i = tid; i < n; i += T) {
        e.sigma[i] = loc[i];
        e.rowid[i] = rid[i];
    }
    if (tid == 0) e.status[0] = s_status;
}

constexpr int UBM = 64;

__device__ __forceinline__ void dmma_16x8x4(double (&c)[4], double a0, double a1, double b0) {
    asm volatile(
        "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 "
        "{%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
        : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
        : "d"(a0), "d"(a1), "d"(b0));
}

// Update v2: 64 x 64 tile, 256 threads.  All global loads of the tile (old
// C rows through sigma, the 16 gathered X rows, the 16 panel columns M) are
// issued back to back into registers and parked in shared memory; the DMMA
// works from shared memory; the result goes out through shared memory with
// coalesced stores.
constexpr int U2T = 256, U2S = 66;   // column stride of the C tile (bank-conflict free)
constexpr size_t U2_SMEM = (64 * U2S + 2 * NB * 68) * sizeof(double);

__global__ void __launch_bounds__(U2T)
gj_update2_kernel(const GjEntry* __restrict__ entries, int kb) {
    const GjEntry e = entries[blockIdx.z];
    const int n = e.n;
    const int k0 = kb * NB;
    if (k0 >= n) return;
    const int nb = min(NB, n - k0);
    const int r0 = blockIdx.x * 64, c0 = blockIdx.y * 64;
    if (r0 >= n || c0 >= n) return;
    if (c0 >= k0 && c0 + 64 <= k0 + nb) return;
    const double* src = buf_of(e, kb & 1);
    double* dst = buf_of(e, (kb + 1) & 1);

    extern __shared__ double u2smem[];
    double (*Cs)[U2S] = reinterpret_cast<double (*)[U2S]>(u2smem);                 // Cs[col][row]
    double (*Ms)[68] = reinterpret_cast<double (*)[68]>(u2smem + 64 * U2S);
    double (*Xs)[68] = reinterpret_cast<double (*)[68]>(u2smem + 64 * U2S + NB * 68);
    __shared__ int srow[64];
    __shared__ int xrow[NB];
    const int tid = threadIdx.x;
    if (tid < 64) srow[tid] = (r0 + tid < n) ? e.sigma[r0 + tid] : 0;
    else if (tid < 64 + NB) {
        const int j = tid - 64;
        xrow[j] = (j < nb) ? e.sigma[k0 + j] : 0;
    }
    __syncthreads();
    double rc[16], rm[4], rx[4];
#pragma unroll
    for (int u = 0; u < 16; ++u) {
        const int idx = tid + u * U2T;
        const int row = idx & 63, col = idx >> 6;
        const int gi = r0 + row, gc = c0 + col;
        double v = 0.0;
        if (gi < n && gc < n && !(gi >= k0 && gi < k0 + nb)) v = src[srow[row] + (size_t)gc * e.ld];
        rc[u] = v;
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const int idx = tid + u * U2T;       // 0..1023
        const int m = idx & 63, j = idx >> 6;
        const int gi = r0 + m;
        rm[u] = (j < nb && gi < n) ? dst[gi + (size_t)(k0 + j) * e.ld] : 0.0;
        const int c = idx >> 4, jj = idx & 15;
        const int gc = c0 + c;
        rx[u] = (jj < nb && gc < n) ? src[xrow[jj] + (size_t)gc * e.ld] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < 16; ++u) {
        const int idx = tid + u * U2T;
        Cs[idx >> 6][idx & 63] = rc[u];
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const int idx = tid + u * U2T;
        Ms[idx >> 6][idx & 63] = rm[u];
        Xs[idx & 15][idx >> 4] = rx[u];
    }
    __syncthreads();

    const int lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int wm = (warp & 1) * 32, wn = (warp >> 1) * 16;
    double acc[2][2][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int jn = 0; jn < 2; ++jn)
#pragma unroll
            for (int v = 0; v < 4; ++v)
                acc[i][jn][v] = Cs[wn + jn * 8 + 2 * t + (v & 1)][wm + i * 16 + g + ((v >> 1) << 3)];
#pragma unroll
    for (int kk = 0; kk < NB; kk += 4) {
        double a[2][2], b[2];
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            a[i][0] = Ms[kk + t][wm + i * 16 + g];
            a[i][1] = Ms[kk + t][wm + i * 16 + g + 8];
        }
#pragma unroll
        for (int jn = 0; jn < 2; ++jn) b[jn] = Xs[kk + t][wn + jn * 8 + g];
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int jn = 0; jn < 2; ++jn) dmma_16x8x4(acc[i][jn], a[i][0], a[i][1], b[jn]);
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int jn = 0; jn < 2; ++jn)
#pragma unroll
            for (int v = 0; v < 4; ++v)
                Cs[wn + jn * 8 + 2 * t + (v & 1)][wm + i * 16 + g + ((v >> 1) << 3)] = acc[i][jn][v];
    __syncthreads();
#pragma unroll
    for (int u = 0; u < 16; ++u) {
        const int idx = tid + u * U2T;
        const int row = idx & 63, col = idx >> 6;
        const int gi = r0 + row, gc = c0 + col;
        if (gi < n && gc < n && !(gc >= k0 && gc < k0 + nb)) dst[gi + (size_t)gc * e.ld] = Cs[col][row];
    }
}

// asynchronous 8-byte global -> shared copy (zero-fill when !pred)
__device__ __forceinline__ void cp_async8(double* sdst, const double* gsrc, bool pred) {
    const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(sdst));
    const int sz = pred ? 8 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" :: "r"(sa), "l"(gsrc), "r"(sz));
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.wait_all;\n" ::: "memory");
}

// ======================================================================
// Two-level blocking.  Outer block of 64 columns (K = [k0, k0 + 64)):
//   4 x { panel on 16 columns of the 64-column window (gj2_panel),
//         rank-16 update of the other window columns (gj2_narrow) }
//   then one rank-64 update of every column outside the window (gj2_trail):
//   new[i, c] = (i in K ? 0 : old[st(i), c]) + sum_{j<64} M64[i, j] old[st(k0 + j), c]
//   with M64 the transformed window and st the composite row map of the
//   four sub-steps.  The window lives in two n x 64 buffers (P), so the
//   sub-steps never touch the rest of the matrix.
constexpr int OB = 64;

__device__ __forceinline__ const double* win_in(const GjEntry& e, int K, int s) {
    return (s == 0) ? buf_of(e, K & 1) + (size_t)(K * OB) * e.ld : e.P + (size_t)(s & 1) * e.ld * OB;
}
__device__ __forceinline__ double* win_out(const GjEntry& e, int s) {
    return e.P + (size_t)((s + 1) & 1) * e.ld * OB;
}

// Row-contiguous layout (RM): the column-major buffer of A is read as the
// row-major B = A^T, so row i of B (column i of A) is contiguous.  A window is
// W columns of B (W = 64 or 128); the window buffers P hold it row-major with
// row stride W.
// Element (row i, window column c) of the window input / output:
// With look-ahead (la = 1) the window buffers and the composite row maps come
// in two sets selected by the parity of the outer step, so the chain of the
// next window never touches what the current trailing update reads.
template <int W>
__device__ __forceinline__ double* win_set_rm(const GjEntry& e, int K, int la) {
    return e.P + (size_t)(la ? 2 * (K & 1) : 0) * e.ld * W;
}
__device__ __forceinline__ int* sigt_set(const GjEntry& e, int K, int la) {
    return e.sigt + (size_t)(la ? 2 * (K & 1) : 0) * e.n;
}
template <int W>
__device__ __forceinline__ const double* win_in_rm(const GjEntry& e, int K, int s, int& lds, int la) {
    if (s == 0) { lds = e.ld; return buf_of(e, K & 1) + (size_t)K * W; }
    lds = W;
    return win_set_rm<W>(e, K, la) + (size_t)(s & 1) * e.ld * W;
}
template <int W>
__device__ __forceinline__ double* win_out_rm(const GjEntry& e, int K, int s, int la) {
    return win_set_rm<W>(e, K, la) + (size_t)((s + 1) & 1) * e.ld * W;
}

// Panel of 16 columns of the 64-column window, one CTA (NW warps) per matrix.
// Each thread keeps R rows of the panel in registers with each row's current
// position (pos); rows never move between threads, a pivot swap only
// relabels two positions.  Pivot choice: largest magnitude among positions
// >= k, ties to the smallest position (partial pivoting as in dgetrf / Eigen
// partialPivLu).  The argmax is exact: a candidate's key is the bit pattern
// of |v| (monotone for non-negative doubles) split into two words, reduced
// with warp max/min reductions, then the smallest position among equal keys.
// Each warp publishes its candidate key and the candidate's whole panel row,
// so one barrier per column hands every thread the pivot and the pivot row.
// The loop is software pipelined: once column j's pivot is known, the next
// column's slot is updated first and its candidate search overlaps the
// update of the other columns.  Rows are eliminated LU-style,
// v -= (f / piv) * pivot_row; the pivot row is rescaled by its one owner.
// The panel columns rotate through the register slots P2_QU at a time, so
// the active column sits in a fixed slot.
constexpr int P2_QU = 2;         // panel columns per unrolled group (rotation step)

struct PivKey {
    unsigned hi, lo;   // hi = 0: no candidate
    int pos;
};

// key of a non-negative magnitude (hi is offset by one so that 0 means none)
__device__ __forceinline__ PivKey piv_key(double a, int pos) {
    if (pos < 0) return PivKey{0u, 0u, -1};
    const unsigned long long b = static_cast<unsigned long long>(__double_as_longlong(a));
    return PivKey{static_cast<unsigned>(b >> 32) + 1u, static_cast<unsigned>(b), pos};
}

// warp-wide best key (every lane gets the result)
__device__ __forceinline__ PivKey warp_best_key(PivKey x) {
    const unsigned H = __reduce_max_sync(0xffffffffu, x.hi);
    const unsigned L = __reduce_max_sync(0xffffffffu, x.hi == H ? x.lo : 0u);
    const bool tie = x.hi == H && x.lo == L && x.pos >= 0;
    const unsigned P = __reduce_min_sync(0xffffffffu, tie ? static_cast<unsigned>(x.pos) : 0xffffffffu);
    return PivKey{H, L, H == 0u ? -1 : static_cast<int>(P)};
}

__device__ __forceinline__ double key_value(const PivKey& k) {
    return __longlong_as_double(static_cast<long long>((static_cast<unsigned long long>(k.hi - 1u) << 32) | k.lo));
}

template <int R, int NW, bool RM, int WIN>
__global__ void __launch_bounds__(NW * 32, 1)
gj2_panel_kernel(const GjEntry* __restrict__ entries, int K, int sub, int la) {
    const GjEntry e = entries[blockIdx.x];
    const int n = e.n;
    const int k0o = K * WIN;
    if (k0o >= n) return;
    const int nb64 = min(WIN, n - k0o);
    const int cs = sub * NB;
    if (cs >= nb64) return;
    const int nb = min(NB, nb64 - cs);
    const int kr0 = k0o + cs;
    int lds = e.ld;
    const double* src = RM ? win_in_rm<WIN>(e, K, sub, lds, la) : win_in(e, K, sub);
    double* dst = RM ? win_out_rm<WIN>(e, K, sub, la) : win_out(e, sub);
    // (row i, window column c) -> element offset
    const size_t rs = RM ? (size_t)lds : 1, cst = RM ? 1 : (size_t)lds;
    const size_t drs = RM ? (size_t)WIN : 1, dcs = RM ? 1 : (size_t)e.ld;
    const int T = blockDim.x, W = T >> 5;
    const bool first = (K == 0 && sub == 0);
    // row-contiguous view: whole 16-byte pairs when the row stride and the column count are even
    const bool vrow = RM && (rs % 2 == 0) && (nb % 2 == 0);

    __shared__ unsigned red_hi[2][NW], red_lo[2][NW];
    __shared__ int red_i[2][NW];
    __shared__ double red_row[2][NW][NB];
    // row labels travel with the rows; kept in shared memory (used at the ends only)
    extern __shared__ int lab_s[];
    int* stv_s = lab_s + n;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    int* sg = RM ? sigt_set(e, K, la) : e.sigt;
    const int* st_in = sg + (size_t)(sub & 1) * n;
    int* st_out = sg + (size_t)((sub + 1) & 1) * n;
    double v[R][NB];
    int pos[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int i = tid + r * T;
        const bool ok = i < n;
        if (RM && vrow) {
            // 16 contiguous doubles of row i in 16-byte pairs
            const double2* rp = reinterpret_cast<const double2*>(src + i * rs + cs);
#pragma unroll
            for (int j = 0; j < NB / 2; ++j) {
                const double2 x = (ok && 2 * j < nb) ? rp[j] : make_double2(0.0, 0.0);
                v[r][2 * j] = x.x;
                v[r][2 * j + 1] = x.y;
            }
        } else {
#pragma unroll
            for (int j = 0; j < NB; ++j) v[r][j] = (ok && j < nb) ? src[i * rs + (size_t)(cs + j) * cst] : 0.0;
        }
        pos[r] = ok ? i : -1;
        if (ok) {
            lab_s[i] = first ? i : e.rowid[i];
            stv_s[i] = (sub == 0) ? i : st_in[i];
        }
    }
    int st_code = 0, st_col = -1;
    if (tid == 0) st_code = first ? 0 : e.status[0];

    // candidate of the first column (slot 0)
    {
        double bv = -1.0;
        int bi = -1;
#pragma unroll
        for (int r = 0; r < R; ++r)
            if (pos[r] >= kr0) better_key(bv, bi, fabs(v[r][0]), pos[r]);
        const PivKey wk = warp_best_key(piv_key(bv, bi));
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const bool mine = wk.pos >= 0 && pos[r] == wk.pos;
            if (__any_sync(0xffffffffu, mine) && mine) {
#pragma unroll
                for (int c = 0; c < NB; ++c) red_row[0][warp][c] = v[r][c];
            }
        }
        if (lane == 0) { red_hi[0][warp] = wk.hi; red_lo[0][warp] = wk.lo; red_i[0][warp] = wk.pos; }
    }

#pragma unroll 1
    for (int g = 0; g < NB / P2_QU; ++g) {
#pragma unroll
        for (int q = 0; q < P2_QU; ++q) {
            const int jj = g * P2_QU + q;
            if (jj < nb) {
                const int k = kr0 + jj;
                const int par = q & 1;
                __syncthreads();
                const PivKey gk = warp_best_key(lane < W ? PivKey{red_hi[par][lane], red_lo[par][lane], red_i[par][lane]}
                                                         : PivKey{0u, 0u, -1});
                const bool have = gk.pos >= 0;
                // positions are unique, so exactly one warp published row gk.pos
                const unsigned own = __ballot_sync(0xffffffffu, have && lane < W && red_i[par][lane] == gk.pos);
                const int ws = own ? __ffs(own) - 1 : 0;
                const int p = have ? gk.pos : k;
                const double* prow = red_row[par][ws];
                double piv = have ? prow[q] : 0.0;
                if (tid == 0 && st_code == 0) {
                    int s = 0;
                    if (!have || !(key_value(gk) < INFINITY)) s = DEV_NONFINITE;
                    else if (key_value(gk) == 0.0) s = DEV_SINGULAR;
                    if (s) { st_code = s; st_col = k; }
                }
                if (piv == 0.0) piv = 1.0;      // the status word records the failure
                const double inv = 1.0 / piv;
                double m[R];
                bool isp[R];
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    m[r] = v[r][q] * inv;
                    isp[r] = have && pos[r] == p;
                    const int pr = pos[r];
                    pos[r] = (pr == p) ? k : (pr == k ? p : pr);
                }
                const bool more = jj + 1 < nb;
                // the next column's slot first, then its candidate search
                if (have) {
                    const double pc = prow[q + 1];
#pragma unroll
                    for (int r = 0; r < R; ++r) v[r][q + 1] = fma(-m[r], pc, v[r][q + 1]);
                }
                PivKey nk{0u, 0u, -1};
                if (more) {
                    double bv = -1.0;
                    int bi = -1;
#pragma unroll
                    for (int r = 0; r < R; ++r)
                        if (pos[r] >= k + 1) better_key(bv, bi, fabs(v[r][q + 1]), pos[r]);
                    nk = warp_best_key(piv_key(bv, bi));
                }
                // the other columns
                if (have) {
#pragma unroll
                    for (int c = 0; c < NB; ++c) {
                        if (c == q || c == q + 1) continue;
                        const double pc = prow[c];
#pragma unroll
                        for (int r = 0; r < R; ++r) v[r][c] = fma(-m[r], pc, v[r][c]);
                    }
                }
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    v[r][q] = -m[r];
                    // the pivot row becomes the scaled pivot row (one thread of one warp)
                    if (__any_sync(0xffffffffu, isp[r]) && isp[r]) {
#pragma unroll
                        for (int c = 0; c < NB; ++c) v[r][c] = (c == q) ? inv : prow[c] * inv;
                    }
                }
                // publish the next column's candidate
                if (more) {
#pragma unroll
                    for (int r = 0; r < R; ++r) {
                        const bool mine = nk.pos >= 0 && pos[r] == nk.pos;
                        if (__any_sync(0xffffffffu, mine) && mine) {
                            // after the group's last column the slots rotate by P2_QU
                            // before the next column reads this row
#pragma unroll
                            for (int c = 0; c < NB; ++c)
                                red_row[par ^ 1][warp][c] = v[r][(q == P2_QU - 1) ? (c + P2_QU) % NB : c];
                        }
                    }
                    if (lane == 0) { red_hi[par ^ 1][warp] = nk.hi; red_lo[par ^ 1][warp] = nk.lo; red_i[par ^ 1][warp] = nk.pos; }
                }
            }
        }
        // rotate the panel columns by P2_QU slots
#pragma unroll
        for (int r = 0; r < R; ++r) {
            double t[P2_QU];
#pragma unroll
            for (int c = 0; c < P2_QU; ++c) t[c] = v[r][c];
#pragma unroll
            for (int c = 0; c < NB - P2_QU; ++c) v[r][c] = v[r][c + P2_QU];
#pragma unroll
            for (int c = 0; c < P2_QU; ++c) v[r][NB - P2_QU + c] = t[c];
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int ps = pos[r];
        if (ps >= 0) {
            if (RM && vrow) {
                double2* wp = reinterpret_cast<double2*>(dst + ps * drs + cs);
#pragma unroll
                for (int j = 0; j < NB / 2; ++j)
                    if (2 * j < nb) wp[j] = make_double2(v[r][2 * j], v[r][2 * j + 1]);
            } else {
#pragma unroll
                for (int j = 0; j < NB; ++j)
                    if (j < nb) dst[ps * drs + (size_t)(cs + j) * dcs] = v[r][j];
            }
            const int i = tid + r * T;
            e.sigma[ps] = i;
            e.rowid[ps] = lab_s[i];
            st_out[ps] = stv_s[i];
        }
    }
    if (tid == 0) {
        e.status[0] = st_code;
        if (st_col >= 0) e.status[1] = st_col;
    }
}

// Panel for orders above one CTA's registers (up to GJ4_CL_MAX x 1024 rows):
// the same elimination as gj2_panel_kernel on the row-contiguous window,
// spread over a thread-block cluster of CL CTAs per matrix.  CTA c keeps rows
// [c RC, (c + 1) RC) of the 16-column panel in registers (RC = R x threads).
// Per column every warp publishes its candidate (key, position) and the
// candidate's panel row in its own shared memory; one cluster barrier
// (arrive = release, wait = acquire) makes them visible cluster-wide; every
// warp then reduces the CL x W candidates read through distributed shared
// memory and reads the pivot row from the owning CTA.  Candidate slots
// alternate by column parity: a slot is rewritten only after every CTA has
// arrived at the barrier that follows its last read.  Every exit depends on
// the matrix only, so it is uniform across the cluster, and a last cluster
// barrier keeps each CTA's shared memory alive until its peers' reads are
// done.  No column rotation here: the active column is picked by a
// compile-time-unrolled select, which keeps every register index static.
constexpr int GJ4_R = 4, GJ4_NW = 8;
constexpr int GJ4_ROWS = GJ4_R * GJ4_NW * 32;        // rows per CTA
constexpr int GJ4_CL_MAX = 8;                       // portable cluster size
// The small cluster panel (any order up to 8 x 384): 2 rows per thread, 6
// warps, at most 170 registers, so that a CTA fits on an SM beside one CTA of
// the trailing update (122 registers x 256 threads) and the panel chain can
// run while the trailing update holds the GPU.
constexpr int GJ4S_R = 2, GJ4S_NW = 6;
constexpr int GJ4S_ROWS = GJ4S_R * GJ4S_NW * 32;

template <int R, int NW, int W, int MINB = 1>
__global__ void __launch_bounds__(NW * 32, MINB)
gj4_panel_kernel(const GjEntry* __restrict__ entries, int K, int sub, int la) {
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    const int CL = (int)cluster.num_blocks();
    const int crank = (int)cluster.block_rank();
    const GjEntry e = entries[blockIdx.x / CL];
    const int n = e.n;
    const int k0o = K * W;
    if (k0o >= n) return;
    const int nb64 = min(W, n - k0o);
    const int cs = sub * NB;
    if (cs >= nb64) return;
    const int nb = min(NB, nb64 - cs);
    const int kr0 = k0o + cs;
    int lds = e.ld;
    const double* src = win_in_rm<W>(e, K, sub, lds, la);
    double* dst = win_out_rm<W>(e, K, sub, la);
    const size_t rs = (size_t)lds;
    constexpr int T = NW * 32;
    constexpr int RC = R * T;
    const int rbase = crank * RC;
    const bool first = (K == 0 && sub == 0);
    const bool vrow = (rs % 2 == 0) && (nb % 2 == 0);

    // candidate key of warp w for column parity p: x = hi, y = lo, z = position
    __shared__ uint4 cand[2][NW];
    __shared__ __align__(16) double cand_row[2][NW][NB];
    __shared__ int lab_s[RC], stv_s[RC];   // labels of this CTA's rows (used at the ends only)

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    int* sg = sigt_set(e, K, la);
    const int* st_in = sg + (size_t)(sub & 1) * n;
    int* st_out = sg + (size_t)((sub + 1) & 1) * n;
    double v[R][NB];
    int pos[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int li = tid + r * T, i = rbase + li;
        const bool ok = i < n;
        if (vrow) {
            const double2* rp = reinterpret_cast<const double2*>(src + (size_t)i * rs + cs);
#pragma unroll
            for (int j = 0; j < NB / 2; ++j) {
                const double2 x = (ok && 2 * j < nb) ? rp[j] : make_double2(0.0, 0.0);
                v[r][2 * j] = x.x;
                v[r][2 * j + 1] = x.y;
            }
        } else {
#pragma unroll
            for (int j = 0; j < NB; ++j) v[r][j] = (ok && j < nb) ? src[(size_t)i * rs + (size_t)(cs + j)] : 0.0;
        }
        pos[r] = ok ? i : -1;
        if (ok) {
            lab_s[li] = first ? i : e.rowid[i];
            stv_s[li] = (sub == 0) ? i : st_in[i];
        }
    }
    const bool leader = crank == 0 && tid == 0;
    int st_code = 0, st_col = -1;
    if (leader) st_code = first ? 0 : e.status[0];

    // this warp's candidate for panel slot `slot` among positions >= `after`, into set `par`
    auto publish = [&](int par, int slot, int after) {
        double bv = -1.0;
        int bi = -1;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            double x = 0.0;
#pragma unroll
            for (int c = 0; c < NB; ++c)
                if (c == slot) x = v[r][c];
            if (pos[r] >= after) better_key(bv, bi, fabs(x), pos[r]);
        }
        const PivKey wk = warp_best_key(piv_key(bv, bi));
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const bool mine = wk.pos >= 0 && pos[r] == wk.pos;
            if (__any_sync(0xffffffffu, mine) && mine) {
#pragma unroll
                for (int c = 0; c < NB; ++c) cand_row[par][warp][c] = v[r][c];
            }
        }
        if (lane == 0) cand[par][warp] = make_uint4(wk.hi, wk.lo, (unsigned)wk.pos, 0u);
    };
    publish(0, 0, kr0);

#pragma unroll 1
    for (int jj = 0; jj < nb; ++jj) {
        const int k = kr0 + jj;
        const int par = jj & 1;
        cluster.sync();
        // best of the cluster's CL x NW candidates, read through distributed shared memory
        PivKey best{0u, 0u, -1};
        int from = 0;                                // cta * NW + warp of best
        for (int idx = lane; idx < CL * NW; idx += 32) {
            const int c = idx / NW, w = idx - c * NW;
            const uint4 x = *cluster.map_shared_rank(&cand[par][w], (unsigned)c);
            const PivKey xk{x.x, x.y, (int)x.z};
            const bool bt = xk.hi > best.hi || (xk.hi == best.hi && xk.lo > best.lo) ||
                            (xk.hi == best.hi && xk.lo == best.lo && xk.pos >= 0 &&
                             (best.pos < 0 || xk.pos < best.pos));
            if (bt) { best = xk; from = idx; }
        }
        const PivKey gk = warp_best_key(best);
        const bool have = gk.pos >= 0;
        // positions are unique: one lane holds the winning candidate
        const unsigned ob = __ballot_sync(0xffffffffu, have && best.pos == gk.pos);
        const int src_idx = __shfl_sync(0xffffffffu, from, ob ? __ffs(ob) - 1 : 0);
        const int oc = src_idx / NW, ow = src_idx - oc * NW;
        const int p = have ? gk.pos : k;
        double pr[NB];
        {
            const double2* prow = reinterpret_cast<const double2*>(
                cluster.map_shared_rank(&cand_row[par][ow][0], (unsigned)oc));
#pragma unroll
            for (int c = 0; c < NB / 2; ++c) {
                const double2 x = have ? prow[c] : make_double2(0.0, 0.0);
                pr[2 * c] = x.x;
                pr[2 * c + 1] = x.y;
            }
        }
        double piv = 0.0;
#pragma unroll
        for (int c = 0; c < NB; ++c)
            if (c == jj) piv = pr[c];
        if (leader && st_code == 0) {
            int s = 0;
            if (!have || !(key_value(gk) < INFINITY)) s = DEV_NONFINITE;
            else if (key_value(gk) == 0.0) s = DEV_SINGULAR;
            if (s) { st_code = s; st_col = k; }
        }
        if (piv == 0.0) piv = 1.0;              // the status word records the failure
        const double inv = 1.0 / piv;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            double vj = 0.0;
#pragma unroll
            for (int c = 0; c < NB; ++c)
                if (c == jj) vj = v[r][c];
            const double m = vj * inv;
            const bool isp = have && pos[r] == p;
            const int pp = pos[r];
            pos[r] = (pp == p) ? k : (pp == k ? p : pp);
            if (have) {
#pragma unroll
                for (int c = 0; c < NB; ++c)
                    if (c != jj) v[r][c] = fma(-m, pr[c], v[r][c]);
            }
#pragma unroll
            for (int c = 0; c < NB; ++c)
                if (c == jj) v[r][c] = -m;
            if (isp) {
                // the pivot row becomes the scaled pivot row
#pragma unroll
                for (int c = 0; c < NB; ++c) v[r][c] = (c == jj) ? inv : pr[c] * inv;
            }
        }
        if (jj + 1 < nb) publish(par ^ 1, jj + 1, k + 1);
    }
    // peers may still be reading this CTA's candidates
    cluster.sync();
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int ps = pos[r];
        if (ps >= 0) {
            if (vrow) {
                double2* wp = reinterpret_cast<double2*>(dst + (size_t)ps * W + cs);
#pragma unroll
                for (int j = 0; j < NB / 2; ++j)
                    if (2 * j < nb) wp[j] = make_double2(v[r][2 * j], v[r][2 * j + 1]);
            } else {
#pragma unroll
                for (int j = 0; j < NB; ++j)
                    if (j < nb) dst[(size_t)ps * W + (cs + j)] = v[r][j];
            }
            const int li = tid + r * T;
            e.sigma[ps] = rbase + li;
            e.rowid[ps] = lab_s[li];
            st_out[ps] = stv_s[li];
        }
    }
    if (leader) {
        e.status[0] = st_code;
        if (st_col >= 0) e.status[1] = st_col;
    }
}

// rank-16 update of the other columns of the 64-column window
__global__ void __launch_bounds__(U2T)
gj2_narrow_kernel(const GjEntry* __restrict__ entries, int K, int sub) {
    const GjEntry e = entries[blockIdx.z];
    const int n = e.n;
    const int k0o = K * OB;
    if (k0o >= n) return;
    const int nb64 = min(OB, n - k0o);
    const int cs = sub * NB;
    if (cs >= nb64) return;
    const int nb = min(NB, nb64 - cs);
    const int kr0 = k0o + cs;
    const int r0 = blockIdx.x * 64;
    if (r0 >= n) return;
    const double* src = win_in(e, K, sub);
    double* dst = win_out(e, sub);

    extern __shared__ double u2smem[];
    double (*Cs)[U2S] = reinterpret_cast<double (*)[U2S]>(u2smem);
    double (*Ms)[68] = reinterpret_cast<double (*)[68]>(u2smem + 64 * U2S);
    double (*Xs)[68] = reinterpret_cast<double (*)[68]>(u2smem + 64 * U2S + NB * 68);
    __shared__ int srow[64];
    __shared__ int xrow[NB];
    const int tid = threadIdx.x;
    if (tid < 64) srow[tid] = (r0 + tid < n) ? e.sigma[r0 + tid] : 0;
    else if (tid < 64 + NB) {
        const int j = tid - 64;
        xrow[j] = (j < nb) ? e.sigma[kr0 + j] : 0;
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < 16; ++u) {
        const int idx = tid + u * U2T;
        const int row = idx & 63, col = idx >> 6;
        const int gi = r0 + row;
        const bool ok = gi < n && col < nb64 && !(gi >= kr0 && gi < kr0 + nb);
        cp_async8(&Cs[col][row], src + (ok ? srow[row] + (size_t)col * e.ld : 0), ok);
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const int idx = tid + u * U2T;
        const int m = idx & 63, j = idx >> 6;
        const int gi = r0 + m;
        const bool okm = j < nb && gi < n;
        cp_async8(&Ms[j][m], dst + (okm ? gi + (size_t)(cs + j) * e.ld : 0), okm);
        const int c = idx >> 4, jj = idx & 15;
        const bool okx = jj < nb && c < nb64;
        cp_async8(&Xs[jj][c], src + (okx ? xrow[jj] + (size_t)c * e.ld : 0), okx);
    }
    cp_async_wait_all();
    __syncthreads();
    const int lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int wm = (warp & 1) * 32, wn = (warp >> 1) * 16;
    double acc[2][2][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int jn = 0; jn < 2; ++jn)
#pragma unroll
            for (int v = 0; v < 4; ++v)
                acc[i][jn][v] = Cs[wn + jn * 8 + 2 * t + (v & 1)][wm + i * 16 + g + ((v >> 1) << 3)];
#pragma unroll
    for (int kk = 0; kk < NB; kk += 4) {
        double a[2][2], b[2];
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            a[i][0] = Ms[kk + t][wm + i * 16 + g];
            a[i][1] = Ms[kk + t][wm + i * 16 + g + 8];
        }
#pragma unroll
        for (int jn = 0; jn < 2; ++jn) b[jn] = Xs[kk + t][wn + jn * 8 + g];
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int jn = 0; jn < 2; ++jn) dmma_16x8x4(acc[i][jn], a[i][0], a[i][1], b[jn]);
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int jn = 0; jn < 2; ++jn)
#pragma unroll
            for (int v = 0; v < 4; ++v)
                Cs[wn + jn * 8 + 2 * t + (v & 1)][wm + i * 16 + g + ((v >> 1) << 3)] = acc[i][jn][v];
    __syncthreads();
#pragma unroll 4
    for (int u = 0; u < 16; ++u) {
        const int idx = tid + u * U2T;
        const int row = idx & 63, col = idx >> 6;
        const int gi = r0 + row;
        if (gi < n && col < nb64 && !(col >= cs && col < cs + nb)) dst[gi + (size_t)col * e.ld] = Cs[col][row];
    }
}

// Trailing rank-64 update, pipelined: old C rows go straight into the DMMA
// accumulators; the 64-deep M / X operands stream through two 16-deep
// shared-memory stages with cp.async, so loads of chunk c+1 overlap the
// tensor-core work on chunk c.
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" :: "n"(N) : "memory"); }

__global__ void __launch_bounds__(U2T, 3)
gj2_trail2_kernel(const GjEntry* __restrict__ entries, int K) {
    const GjEntry e = entries[blockIdx.z];
    const int n = e.n;
    const int k0 = K * OB;
    if (k0 >= n) return;
    const int nb64 = min(OB, n - k0);
    const int nsub = (nb64 + NB - 1) / NB;
    const int r0 = blockIdx.x * 64, c0 = blockIdx.y * 64;
    if (r0 >= n || c0 >= n) return;
    const double* src = buf_of(e, K & 1);
    double* dst = buf_of(e, (K + 1) & 1);
    const double* Mw = e.P + (size_t)(nsub & 1) * e.ld * OB;
    const int* st = e.sigt + (size_t)(nsub & 1) * n;
    const int tid = threadIdx.x;
    if (c0 == k0) {
        for (int idx = tid; idx < 64 * 64; idx += U2T) {
            const int row = idx & 63, col = idx >> 6;
            const int gi = r0 + row;
            if (gi < n && col < nb64) dst[gi + (size_t)(c0 + col) * e.ld] = Mw[gi + (size_t)col * e.ld];
        }
        return;
    }
    __shared__ double Ms[2][NB][68];
    __shared__ double Xs[2][NB][68];
    __shared__ int srow[64];
    __shared__ int xrow[64];
    if (tid < 64) srow[tid] = (r0 + tid < n) ? st[r0 + tid] : 0;
    else if (tid < 128) {
        const int j = tid - 64;
        xrow[j] = (j < nb64) ? st[k0 + j] : 0;
    }
    __syncthreads();
    auto load_chunk = [&](int ch, int buf) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int idx = tid + u * U2T;          // 0..1023
            const int m = idx & 63, jj = idx >> 6;  // Ms[jj][m]
            const int j = ch * NB + jj;
            const int gi = r0 + m;
            const bool okm = j < nb64 && gi < n;
            cp_async8(&Ms[buf][jj][m], Mw + (okm ? gi + (size_t)j * e.ld : 0), okm);
            const int c = idx >> 4, jx = idx & 15;  // Xs[jx][c]
            const int jg = ch * NB + jx;
            const int gc = c0 + c;
            const bool okx = jg < nb64 && gc < n;
            cp_async8(&Xs[buf][jx][c], src + (okx ? xrow[jg] + (size_t)gc * e.ld : 0), okx);
        }
        cp_async_commit();
    };
    load_chunk(0, 0);
    const int lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int wm = (warp & 1) * 32, wn = (warp >> 1) * 16;
    double acc[2][2][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int jn = 0; jn < 2; ++jn)
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                const int rl = wm + i * 16 + g + ((v >> 1) << 3);
                const int gi = r0 + rl;
                const int gc = c0 + wn + jn * 8 + 2 * t + (v & 1);
                double old = 0.0;
                if (gi < n && gc < n && !(gi >= k0 && gi < k0 + nb64)) old = src[srow[rl] + (size_t)gc * e.ld];
                acc[i][jn][v] = old;
            }
    const int nch = nsub;
    for (int ch = 0; ch < nch; ++ch) {
        const int buf = ch & 1;
        if (ch + 1 < nch) {
            load_chunk(ch + 1, buf ^ 1);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < NB; kk += 4) {
            double a[2][2], b[2];
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                a[i][0] = Ms[buf][kk + t][wm + i * 16 + g];
                a[i][1] = Ms[buf][kk + t][wm + i * 16 + g + 8];
            }
#pragma unroll
            for (int jn = 0; jn < 2; ++jn) b[jn] = Xs[buf][kk + t][wn + jn * 8 + g];
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int jn = 0; jn < 2; ++jn) dmma_16x8x4(acc[i][jn], a[i][0], a[i][1], b[jn]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int jn = 0; jn < 2; ++jn)
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                const int gi = r0 + wm + i * 16 + g + ((v >> 1) << 3);
                const int gc = c0 + wn + jn * 8 + 2 * t + (v & 1);
                if (gi < n && gc < n) dst[gi + (size_t)gc * e.ld] = acc[i][jn][v];
            }
}

// ---------------------------------------------------------------------------
// Row-contiguous (RM) narrow and trailing updates.  Every operand row is a
// contiguous run: the pivot rows of the old matrix, the rows of the
// transformed window and the C tile rows are copied with 16-byte cp.async
// when the row stride is even (8-byte copies otherwise).

__device__ __forceinline__ void cp_async16(double* sdst, const double* gsrc, bool pred) {
    const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(sdst));
    const int sz = pred ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" :: "r"(sa), "l"(gsrc), "r"(sz));
}

constexpr int N3S = 20;      // row stride of the 64 x 16 multiplier tile (= 4 mod 16)
constexpr int T3R = 68;      // row stride of the 64-wide tiles (= 4 mod 16)
constexpr size_t NARROW3_SMEM = (64 * T3R + 64 * N3S + NB * T3R) * sizeof(double);

// rank-16 update of the other columns of the W-column window (RM layout),
// one 64 x 64 tile (rows blockIdx.x, window columns blockIdx.y) per CTA:
//   out[i, c] = (i a pivot position of this panel ? 0 : in[sigma(i), c])
//               + sum_j Mp[i, j] in[sigma(kr0 + j), c]
template <int W>
__global__ void __launch_bounds__(U2T)
gj3_narrow_kernel(const GjEntry* __restrict__ entries, int K, int sub, int la) {
    const GjEntry e = entries[blockIdx.z];
    const int n = e.n;
    const int k0o = K * W;
    if (k0o >= n) return;
    const int nbw = min(W, n - k0o);
    const int cs = sub * NB;
    if (cs >= nbw) return;
    const int nb = min(NB, nbw - cs);
    const int kr0 = k0o + cs;
    const int r0 = blockIdx.x * 64;
    const int cw = blockIdx.y * 64;           // first window column of this tile
    if (r0 >= n || cw >= nbw) return;
    const int nb64 = min(64, nbw - cw);       // window columns of this tile
    int lds;
    const double* src = win_in_rm<W>(e, K, sub, lds, la) + cw;
    double* dst = win_out_rm<W>(e, K, sub, la);
    // 16-byte rows need an even stride; the big buffer also needs whole pairs inside the window
    const bool v16 = (lds % 2 == 0) && (sub > 0 || nbw % 2 == 0);

    extern __shared__ double n3smem[];
    double (*Cs)[T3R] = reinterpret_cast<double (*)[T3R]>(n3smem);
    double (*Ms)[N3S] = reinterpret_cast<double (*)[N3S]>(n3smem + 64 * T3R);
    double (*Xs)[T3R] = reinterpret_cast<double (*)[T3R]>(n3smem + 64 * T3R + 64 * N3S);
    __shared__ int srow[64];
    __shared__ int xrow[NB];
    const int tid = threadIdx.x;
    if (tid < 64) srow[tid] = (r0 + tid < n) ? e.sigma[r0 + tid] : 0;
    else if (tid < 64 + NB) {
        const int j = tid - 64;
        xrow[j] = (j < nb) ? e.sigma[kr0 + j] : 0;
    }
    __syncthreads();
    if (v16) {
#pragma unroll
        for (int u = 0; u < 8; ++u) {              // C: 64 rows x 32 pairs
            const int idx = tid + u * U2T;
            const int row = idx >> 5, c = 2 * (idx & 31);
            const int gi = r0 + row;
            const bool ok = gi < n && c < nb64 && !(gi >= kr0 && gi < kr0 + nb);
            cp_async16(&Cs[row][c], src + (ok ? (size_t)srow[row] * lds + c : 0), ok);
        }
#pragma unroll
        for (int u = 0; u < 2; ++u) {              // X: 16 pivot rows x 32 pairs
            const int idx = tid + u * U2T;
            const int j = idx >> 5, c = 2 * (idx & 31);
            const bool ok = j < nb && c < nb64;
            cp_async16(&Xs[j][c], src + (ok ? (size_t)xrow[j] * lds + c : 0), ok);
        }
    } else {
#pragma unroll 4
        for (int u = 0; u < 16; ++u) {
            const int idx = tid + u * U2T;
            const int row = idx >> 6, c = idx & 63;
            const int gi = r0 + row;
            const bool ok = gi < n && c < nb64 && !(gi >= kr0 && gi < kr0 + nb);
            cp_async8(&Cs[row][c], src + (ok ? (size_t)srow[row] * lds + c : 0), ok);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int idx = tid + u * U2T;
            const int j = idx >> 6, c = idx & 63;
            const bool ok = j < nb && c < nb64;
            cp_async8(&Xs[j][c], src + (ok ? (size_t)xrow[j] * lds + c : 0), ok);
        }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {                  // Mp: 64 rows x 16 (panel output, stride W)
        const int idx = tid + u * U2T;
        const int m = idx >> 4, j = idx & 15;
        const int gi = r0 + m;
        const bool ok = gi < n && j < nb;
        cp_async8(&Ms[m][j], dst + (ok ? (size_t)gi * W + cs + j : 0), ok);
    }
    cp_async_wait_all();
    __syncthreads();
    const int lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int wm = (warp & 1) * 32, wn = (warp >> 1) * 16;
    double acc[2][2][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int jn = 0; jn < 2; ++jn)
#pragma unroll
            for (int v = 0; v < 4; ++v)
                acc[i][jn][v] = Cs[wm + i * 16 + g + ((v >> 1) << 3)][wn + jn * 8 + 2 * t + (v & 1)];
#pragma unroll
    for (int kk = 0; kk < NB; kk += 4) {
        double a[2][2], b[2];
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            a[i][0] = Ms[wm + i * 16 + g][kk + t];
            a[i][1] = Ms[wm + i * 16 + g + 8][kk + t];
        }
#pragma unroll
        for (int jn = 0; jn < 2; ++jn) b[jn] = Xs[kk + t][wn + jn * 8 + g];
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int jn = 0; jn < 2; ++jn) dmma_16x8x4(acc[i][jn], a[i][0], a[i][1], b[jn]);
    }
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int jn = 0; jn < 2; ++jn)
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                const int gi = r0 + wm + i * 16 + g + ((v >> 1) << 3);
                const int c = wn + jn * 8 + 2 * t + (v & 1);
                if (gi < n && c < nb64 && !(cw + c >= cs && cw + c < cs + nb))
                    dst[(size_t)gi * W + cw + c] = acc[i][jn][v];
            }
}

// rank-64 update of every column tile outside the window (RM layout), one
// 128 x 64 tile per CTA, 8 warps of 32 x 32:
//   new[i, c] = (i in the window rows ? 0 : old[st(i), c]) + sum_j M[i, j] old[st(k0 + j), c]
// M = the transformed window (row-major, stride OB); the window's own column
// tile is copied from M.  The k dimension arrives in four 16-wide cp.async
// groups so the first DMMAs start before the whole tile has landed.
constexpr int T3M = 128;
constexpr size_t TRAIL3_SMEM = (T3M * T3R + OB * T3R) * sizeof(double);

// cols: -1 every column tile; t >= 0 only tile t; -2 - t every tile but t
__global__ void __launch_bounds__(U2T, 2)
gj3_trail_kernel(const GjEntry* __restrict__ entries, int K, int la, int cols) {
    const GjEntry e = entries[blockIdx.z];
    const int n = e.n;
    const int k0 = K * OB;
    if (k0 >= n) return;
    const int nb64 = min(OB, n - k0);
    const int nsub = (nb64 + NB - 1) / NB;
    int ct = blockIdx.y;
    if (cols >= 0) ct = cols;
    else if (cols <= -2 && ct >= -2 - cols) ++ct;
    const int r0 = blockIdx.x * T3M, c0 = ct * 64;
    if (r0 >= n || c0 >= n) return;
    const size_t ld = e.ld;
    const double* src = buf_of(e, K & 1);
    double* dst = buf_of(e, (K + 1) & 1);
    const double* Mw = win_set_rm<OB>(e, K, la) + (size_t)(nsub & 1) * e.ld * OB;
    const int* st = sigt_set(e, K, la) + (size_t)(nsub & 1) * n;
    const int tid = threadIdx.x;
    if (c0 == k0) {
        for (int idx = tid; idx < T3M * 64; idx += U2T) {
            const int row = idx >> 6, col = idx & 63;
            const int gi = r0 + row;
            if (gi < n && col < nb64) dst[gi * ld + k0 + col] = Mw[(size_t)gi * OB + col];
        }
        return;
    }
    const bool v16 = (ld % 2 == 0);          // n even: pairs never straddle a row end
    const bool m16 = (nb64 % 2 == 0);        // whole pairs inside the window
    extern __shared__ double t3smem[];
    double (*Ms)[T3R] = reinterpret_cast<double (*)[T3R]>(t3smem);
    double (*Xs)[T3R] = reinterpret_cast<double (*)[T3R]>(t3smem + T3M * T3R);
    __shared__ int srow[T3M];
    __shared__ int xrow[OB];
    if (tid < T3M) srow[tid] = (r0 + tid < n) ? st[r0 + tid] : 0;
    else if (tid < T3M + OB) {
        const int j = tid - T3M;
        xrow[j] = (j < nb64) ? st[k0 + j] : 0;
    }
    __syncthreads();
#pragma unroll
    for (int ch = 0; ch < 4; ++ch) {
        if (m16) {
#pragma unroll
            for (int u = 0; u < 4; ++u) {          // M: 128 rows x 8 pairs of this chunk
                const int idx = tid + u * U2T;
                const int m = idx >> 3, j = ch * NB + 2 * (idx & 7);
                const int gi = r0 + m;
                const bool ok = gi < n && j < nb64;
                cp_async16(&Ms[m][j], Mw + (ok ? (size_t)gi * OB + j : 0), ok);
            }
        } else {
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int idx = tid + u * U2T;
                const int m = idx >> 4, j = ch * NB + (idx & 15);
                const int gi = r0 + m;
                const bool ok = gi < n && j < nb64;
                cp_async8(&Ms[m][j], Mw + (ok ? (size_t)gi * OB + j : 0), ok);
            }
        }
        if (v16) {
#pragma unroll
            for (int u = 0; u < 2; ++u) {          // X: 16 pivot rows x 32 pairs
                const int idx = tid + u * U2T;
                const int j = ch * NB + (idx >> 5), c = 2 * (idx & 31);
                const bool ok = j < nb64 && c0 + c < n;
                cp_async16(&Xs[j][c], src + (ok ? (size_t)xrow[j] * ld + c0 + c : 0), ok);
            }
        } else {
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int idx = tid + u * U2T;
                const int j = ch * NB + (idx >> 6), c = idx & 63;
                const bool ok = j < nb64 && c0 + c < n;
                cp_async8(&Xs[j][c], src + (ok ? (size_t)xrow[j] * ld + c0 + c : 0), ok);
            }
        }
        cp_async_commit();
    }
    const int lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int wm = (warp & 3) * 32, wn = (warp >> 2) * 32;
    double acc[2][4][4];
    // C tile straight from the old matrix into the accumulators
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int rl = wm + i * 16 + g + 8 * h;
            const int gi = r0 + rl;
            const bool rok = gi < n && !(gi >= k0 && gi < k0 + nb64);
            const double* rowp = src + (size_t)srow[rl] * ld + c0;
#pragma unroll
            for (int jn = 0; jn < 4; ++jn) {
                const int c = wn + jn * 8 + 2 * t;
                double x0 = 0.0, x1 = 0.0;
                if (rok && c0 + c < n) {
                    if (v16) {
                        const double2 p2 = *reinterpret_cast<const double2*>(rowp + c);
                        x0 = p2.x; x1 = p2.y;
                    } else {
                        x0 = rowp[c];
                        if (c0 + c + 1 < n) x1 = rowp[c + 1];
                    }
                }
                acc[i][jn][2 * h] = x0;
                acc[i][jn][2 * h + 1] = x1;
            }
        }
#pragma unroll
    for (int ch = 0; ch < 4; ++ch) {
        if (ch == 0) cp_async_wait<3>();
        else if (ch == 1) cp_async_wait<2>();
        else if (ch == 2) cp_async_wait<1>();
        else cp_async_wait<0>();
        __syncthreads();
        if (ch < nsub) {
#pragma unroll
            for (int kq = 0; kq < NB; kq += 4) {
                const int kk = ch * NB + kq;
                double a[2][2], b[4];
#pragma unroll
                for (int i = 0; i < 2; ++i) {
                    a[i][0] = Ms[wm + i * 16 + g][kk + t];
                    a[i][1] = Ms[wm + i * 16 + g + 8][kk + t];
                }
#pragma unroll
                for (int jn = 0; jn < 4; ++jn) b[jn] = Xs[kk + t][wn + jn * 8 + g];
#pragma unroll
                for (int i = 0; i < 2; ++i)
#pragma unroll
                    for (int jn = 0; jn < 4; ++jn) dmma_16x8x4(acc[i][jn], a[i][0], a[i][1], b[jn]);
            }
        }
    }
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int gi = r0 + wm + i * 16 + g + 8 * h;
            if (gi >= n) continue;
            double* rowp = dst + (size_t)gi * ld + c0;
#pragma unroll
            for (int jn = 0; jn < 4; ++jn) {
                const int c = wn + jn * 8 + 2 * t;
                if (c0 + c >= n) continue;
                if (v16) {
                    *reinterpret_cast<double2*>(rowp + c) = make_double2(acc[i][jn][2 * h], acc[i][jn][2 * h + 1]);
                } else {
                    rowp[c] = acc[i][jn][2 * h];
                    if (c0 + c + 1 < n) rowp[c + 1] = acc[i][jn][2 * h + 1];
                }
            }
        }
}

// rank-128 update for 128-column windows (RM layout), one 128 x 64 C tile per
// CTA, 8 warps of 32 x 32 DMMA, 2 CTAs per SM.  Twice the flops of the
// rank-64 update for the same C-tile load and store.  The k dimension (the
// window's columns) streams through a two-stage cp.async ring of 32-column
// stages (M: 128 x 32, X: 32 x 64), so a stage lands while the previous one
// is multiplied; the C tile goes straight from the old matrix into the
// accumulators meanwhile.
// Column tiles: blockIdx.y + ct_lo, moved past [skip_lo, skip_lo + skip_n).
constexpr int T3K = 32;                      // window columns per stage
constexpr int T3KS = 36;                     // row stride of the M stage (= 4 mod 16)
constexpr int T3STAGE = T3M * T3KS + T3K * T3R;
constexpr size_t TRAIL128_SMEM = 2 * (size_t)T3STAGE * sizeof(double);

__global__ void __launch_bounds__(U2T, 2)
gj3_trail128_kernel(const GjEntry* __restrict__ entries, int K, int la, int ct_lo, int skip_lo, int skip_n) {
    constexpr int W = 128;
    const GjEntry e = entries[blockIdx.z];
    const int n = e.n;
    const int k0 = K * W;
    if (k0 >= n) return;
    const int nbw = min(W, n - k0);
    const int nsub = (nbw + NB - 1) / NB;
    int ct = ct_lo + (int)blockIdx.y;
    if (skip_n > 0 && ct >= skip_lo) ct += skip_n;
    const int r0 = blockIdx.x * T3M, c0 = ct * 64;
    if (r0 >= n || c0 >= n) return;
    const size_t ld = e.ld;
    const double* src = buf_of(e, K & 1);
    double* dst = buf_of(e, (K + 1) & 1);
    const double* Mw = win_set_rm<W>(e, K, la) + (size_t)(nsub & 1) * e.ld * W;
    const int* st = sigt_set(e, K, la) + (size_t)(nsub & 1) * n;
    const int tid = threadIdx.x;
    if (c0 >= k0 && c0 < k0 + nbw) {
        // a column tile of the window itself: the transformed window
        const int cw = c0 - k0;
        for (int idx = tid; idx < T3M * 64; idx += U2T) {
            const int row = idx >> 6, col = idx & 63;
            const int gi = r0 + row;
            if (gi < n && cw + col < nbw) dst[gi * ld + c0 + col] = Mw[(size_t)gi * W + cw + col];
        }
        return;
    }
    const bool v16 = (ld % 2 == 0);          // n even: pairs never straddle a row end
    const bool m16 = (nbw % 2 == 0);         // whole pairs inside the window
    extern __shared__ double t128smem[];
    __shared__ int srow[T3M];
    __shared__ int xrow[W];
    if (tid < T3M) srow[tid] = (r0 + tid < n) ? st[r0 + tid] : 0;
    else if (tid < T3M + W) {
        const int j = tid - T3M;
        xrow[j] = (j < nbw) ? st[k0 + j] : 0;
    }
    __syncthreads();
    const int nch = (nbw + T3K - 1) / T3K;
    // stage s: M rows at t128smem + s * T3STAGE (stride T3KS), X rows after them (stride T3R)
    auto issue = [&](int ch) {
        double* Ms = t128smem + (size_t)(ch & 1) * T3STAGE;
        double* Xs = Ms + T3M * T3KS;
        const int kb = ch * T3K;
        if (m16) {
#pragma unroll
            for (int u = 0; u < 8; ++u) {          // M: 128 rows x 16 pairs
                const int idx = tid + u * U2T;
                const int m = idx >> 4, j = 2 * (idx & 15);
                const int gi = r0 + m;
                const bool ok = gi < n && kb + j < nbw;
                cp_async16(Ms + m * T3KS + j, Mw + (ok ? (size_t)gi * W + kb + j : 0), ok);
            }
        } else {
#pragma unroll 4
            for (int u = 0; u < 16; ++u) {
                const int idx = tid + u * U2T;
                const int m = idx >> 5, j = idx & 31;
                const int gi = r0 + m;
                const bool ok = gi < n && kb + j < nbw;
                cp_async8(Ms + m * T3KS + j, Mw + (ok ? (size_t)gi * W + kb + j : 0), ok);
            }
        }
        if (v16) {
#pragma unroll
            for (int u = 0; u < 4; ++u) {          // X: 32 pivot rows x 32 pairs
                const int idx = tid + u * U2T;
                const int j = idx >> 5, c = 2 * (idx & 31);
                const bool ok = kb + j < nbw && c0 + c < n;
                cp_async16(Xs + j * T3R + c, src + (ok ? (size_t)xrow[kb + j] * ld + c0 + c : 0), ok);
            }
        } else {
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int idx = tid + u * U2T;
                const int j = idx >> 6, c = idx & 63;
                const bool ok = kb + j < nbw && c0 + c < n;
                cp_async8(Xs + j * T3R + c, src + (ok ? (size_t)xrow[kb + j] * ld + c0 + c : 0), ok);
            }
        }
        cp_async_commit();
    };
    const int lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int wm = (warp & 3) * 32, wn = (warp >> 2) * 32;
    double acc[2][4][4];
    // C tile straight from the old matrix into the accumulators: issued
    // first, its HBM latency is the longest; the first two k stages follow
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int rl = wm + i * 16 + g + 8 * h;
            const int gi = r0 + rl;
            const bool rok = gi < n && !(gi >= k0 && gi < k0 + nbw);
            const double* rowp = src + (size_t)srow[rl] * ld + c0;
#pragma unroll
            for (int jn = 0; jn < 4; ++jn) {
                const int c = wn + jn * 8 + 2 * t;
                double x0 = 0.0, x1 = 0.0;
                if (rok && c0 + c < n) {
                    if (v16) {
                        const double2 p2 = *reinterpret_cast<const double2*>(rowp + c);
                        x0 = p2.x; x1 = p2.y;
                    } else {
                        x0 = rowp[c];
                        if (c0 + c + 1 < n) x1 = rowp[c + 1];
                    }
                }
                acc[i][jn][2 * h] = x0;
                acc[i][jn][2 * h + 1] = x1;
            }
        }
    issue(0);
    if (nch > 1) issue(1);
#pragma unroll 1
    for (int ch = 0; ch < nch; ++ch) {
        if (ch + 1 < nch) cp_async_wait<1>();
        else cp_async_wait<0>();
        __syncthreads();
        const double* Ms = t128smem + (size_t)(ch & 1) * T3STAGE;
        const double* Xs = Ms + T3M * T3KS;
#pragma unroll
        for (int kq = 0; kq < T3K; kq += 4) {
            double a[2][2], b[4];
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                a[i][0] = Ms[(wm + i * 16 + g) * T3KS + kq + t];
                a[i][1] = Ms[(wm + i * 16 + g + 8) * T3KS + kq + t];
            }
#pragma unroll
            for (int jn = 0; jn < 4; ++jn) b[jn] = Xs[(kq + t) * T3R + wn + jn * 8 + g];
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int jn = 0; jn < 4; ++jn) dmma_16x8x4(acc[i][jn], a[i][0], a[i][1], b[jn]);
        }
        if (ch + 2 < nch) {
            __syncthreads();                         // every warp is done with this stage
            issue(ch + 2);
        }
    }
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int gi = r0 + wm + i * 16 + g + 8 * h;
            if (gi >= n) continue;
            double* rowp = dst + (size_t)gi * ld + c0;
#pragma unroll
            for (int jn = 0; jn < 4; ++jn) {
                const int c = wn + jn * 8 + 2 * t;
                if (c0 + c >= n) continue;
                if (v16) {
                    *reinterpret_cast<double2*>(rowp + c) = make_double2(acc[i][jn][2 * h], acc[i][jn][2 * h + 1]);
                } else {
                    rowp[c] = acc[i][jn][2 * h];
                    if (c0 + c + 1 < n) rowp[c + 1] = acc[i][jn][2 * h + 1];
                }
            }
        }
}

constexpr int FT = 32;

__global__ void __launch_bounds__(FT * 8)
gj_finalize_kernel(const GjEntry* __restrict__ entries, int wstep, int symmetrize, int rm) {
    // wstep: columns per block step (16 single-level, 64 or 128 two-level)
    const GjEntry e = entries[blockIdx.z];
    const int n = e.n;
    const int i0 = blockIdx.x * FT, j0 = blockIdx.y * FT;
    if (i0 >= n || j0 >= n) return;
    // the result of the last block step lives in buffer (number of steps of this matrix) % 2
    const int steps = (n + wstep - 1) / wstep;
    const double* X = buf_of(e, steps & 1);

    __shared__ int pi_i[FT], pi_j[FT];
    __shared__ double T1[FT][FT + 1];
    __shared__ double T2[FT][FT + 1];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;   // 32 x 8
    // pi = inverse of rowid: pi[rowid[r]] = r.  Scan for the 32 + 32 labels we need.
    if (threadIdx.x < 64) {
        // filled below by the scan
    }
    for (int r = threadIdx.x; r < n; r += blockDim.x) {
        const int id = e.rowid[r];
        if (id >= i0 && id < i0 + FT) pi_i[id - i0] = r;
        if (id >= j0 && id < j0 + FT) pi_j[id - j0] = r;
    }
    __syncthreads();
    // column-major layout: inv[i][j] = X[i][pi(j)]
    // row-contiguous layout (X holds inv(A^T) row-major): inv[i][j] = X[j * ld + pi(i)]
    // T1[a][b] = inv[i0 + a][j0 + b],  T2[a][b] = inv[j0 + a][i0 + b]
    for (int b = ty; b < FT; b += 8) {
        const int a = tx;
        if (j0 + b < n && i0 + a < n)
            T1[a][b] = rm ? X[(size_t)(j0 + b) * e.ld + pi_i[a]] : X[(i0 + a) + (size_t)pi_j[b] * e.ld];
        if (symmetrize && i0 + b < n && j0 + a < n)
            T2[a][b] = rm ? X[(size_t)(i0 + b) * e.ld + pi_j[a]] : X[(j0 + a) + (size_t)pi_i[b] * e.ld];
    }
    __syncthreads();
    for (int b = ty; b < FT; b += 8) {
        const int a = tx;
        const int i = i0 + a, j = j0 + b;
        if (i < n && j < n) {
            double v = T1[a][b];
            if (symmetrize) v = 0.5 * (v + T2[b][a]);
            e.out[i + (size_t)j * e.ldo] = v;
        }
    }
}

// Cluster shape of the panel for orders above one CTA: CTAs per matrix.
int gj4_cluster_size(int nmax, int pcfg) {
    const int rows = pcfg == GJ_PANEL_SMALL_CLUSTER ? GJ4S_ROWS : GJ4_ROWS;
    return (nmax + rows - 1) / rows;
}

// pcfg GJ_PANEL_SHAPES: the cluster panel (RM only), gj4_cluster_size CTAs per matrix;
// pcfg GJ_PANEL_SMALL_CLUSTER: the small cluster panel (RM only);
// W: window width (64 for the column-major scheme)
template <bool RM, int W>
int launch_panel(int pcfg, int count, int pt, size_t smem, cudaStream_t stream, const GjEntry* ent, int K, int sub,
                 int la, int nmax = 0) {
    if (RM && (pcfg == GJ_PANEL_SHAPES || pcfg == GJ_PANEL_SMALL_CLUSTER)) {
        const bool small = pcfg == GJ_PANEL_SMALL_CLUSTER;
        const int cl = gj4_cluster_size(nmax, pcfg);
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)(count * cl), 1, 1);
        cfg.blockDim = dim3((small ? GJ4S_NW : GJ4_NW) * 32, 1, 1);
        cfg.dynamicSmemBytes = 0;
        cfg.stream = stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = (unsigned)cl;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        if (small)
            SCATT_CUDA_TRY(cudaLaunchKernelEx(&cfg, gj4_panel_kernel<GJ4S_R, GJ4S_NW, W, 2>, ent, K, sub, la));
        else
            SCATT_CUDA_TRY(cudaLaunchKernelEx(&cfg, gj4_panel_kernel<GJ4_R, GJ4_NW, W>, ent, K, sub, la));
        return SCATT_OK;
    }
    switch (pcfg) {
        case 0: gj2_panel_kernel<1, 8, RM, W><<<count, pt, smem, stream>>>(ent, K, sub, la); break;
        case 1: gj2_panel_kernel<2, 8, RM, W><<<count, pt, smem, stream>>>(ent, K, sub, la); break;
        case 2: gj2_panel_kernel<3, 8, RM, W><<<count, pt, smem, stream>>>(ent, K, sub, la); break;
        case 3: gj2_panel_kernel<3, 12, RM, W><<<count, pt, smem, stream>>>(ent, K, sub, la); break;
        default: gj2_panel_kernel<5, 8, RM, W><<<count, pt, smem, stream>>>(ent, K, sub, la); break;
    }
    return SCATT_OK;
}

// Side stream (highest priority) and two events per (device, main stream)
// for the look-ahead of the row-contiguous inverse, created on first use.
// Inverses enqueued on different streams (the phase groups of a scan) get
// different side streams, so their look-ahead chains do not queue behind
// one another.  The enqueueing of one inverse holds the mutex, so its event
// record / wait pairs cannot interleave with another thread's.
struct LookAhead {
    cudaStream_t side = nullptr;
    cudaEvent_t ev_main = nullptr, ev_side = nullptr;
};
std::mutex g_la_mutex;
std::map<std::pair<int, cudaStream_t>, LookAhead> g_la;

int look_ahead_resources(cudaStream_t main, LookAhead** out) {
    int dev = 0;
    SCATT_CUDA_TRY(cudaGetDevice(&dev));
    LookAhead& r = g_la[std::make_pair(dev, main)];
    if (!r.side) {
        int lo = 0, hi = 0;
        SCATT_CUDA_TRY(cudaDeviceGetStreamPriorityRange(&lo, &hi));
        SCATT_CUDA_TRY(cudaStreamCreateWithPriority(&r.side, cudaStreamNonBlocking, hi));
        SCATT_CUDA_TRY(cudaEventCreateWithFlags(&r.ev_main, cudaEventDisableTiming));
        SCATT_CUDA_TRY(cudaEventCreateWithFlags(&r.ev_side, cudaEventDisableTiming));
    }
    *out = &r;
    return SCATT_OK;
}

// panel shape (rows per thread x warps): 1x8 (n <= 256), 2x8 (<= 512),
// 3x8 (<= 768), 3x12 (<= 1152), 5x8 (<= 1280); `force` (>= 0) picks one
// that holds nmax.  pt = the threads of the launch: ceil(nmax / rows) rounded
// up to whole warps, at most the shape's warps since nmax <= its capacity.
int panel_shape(int nmax, int& pcfg, int& pt, int force = -1) {
    if (force == GJ_PANEL_SMALL_CLUSTER) {
        if (nmax > GJ4S_ROWS * GJ4_CL_MAX) {
            set_last_error("inverse: the small cluster panel does not hold order " + std::to_string(nmax));
            return SCATT_ERR_ARG;
        }
        pcfg = force;
        pt = GJ4S_NW * 32;
        return SCATT_OK;
    }
    if (nmax > gj_panel_capacity(GJ_PANEL_SHAPES - 1)) {
        // beyond one CTA: the cluster panel
        if (force >= 0 && force != GJ_PANEL_SHAPES) {
            set_last_error("inverse: panel shape " + std::to_string(force) + " does not hold order " +
                           std::to_string(nmax));
            return SCATT_ERR_ARG;
        }
        if (nmax > GJ4_ROWS * GJ4_CL_MAX) {
            set_last_error("inverse: order " + std::to_string(nmax) + " exceeds the cluster panel limit " +
                           std::to_string(GJ4_ROWS * GJ4_CL_MAX));
            return SCATT_ERR_SIZE;
        }
        pcfg = GJ_PANEL_SHAPES;
        pt = GJ4_NW * 32;
        return SCATT_OK;
    }
    if (force >= 0) {
        if (force >= GJ_PANEL_SHAPES || nmax > gj_panel_capacity(force)) {
            set_last_error("inverse: panel shape " + std::to_string(force) + " does not hold order " +
                           std::to_string(nmax));
            return SCATT_ERR_ARG;
        }
        pcfg = force;
    } else {
        pcfg = nmax <= 256 ? 0 : nmax <= 512 ? 1 : nmax <= 768 ? 2 : nmax <= 1152 ? 3 : 4;
    }
    const int prows = pcfg == 0 ? 1 : pcfg == 1 ? 2 : pcfg <= 3 ? 3 : 5;
    pt = 32 * (((nmax + prows - 1) / prows + 31) / 32);
    return SCATT_OK;
}

// autotuned choices, keyed by (device, order, batch)
std::mutex g_tune_mutex;
std::map<std::tuple<int, int, int>, InverseTune> g_tune;

// Kernel attributes are per device: one flag bit per device and scheme.
std::mutex g_attr_mutex;
unsigned long long g_attr_done[3] = {0, 0, 0};

// Runs set() once per (scheme, current device); returns its status.
template <class F>
int once_per_device(int scheme, F set) {
    int dev = 0;
    SCATT_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) {
        set_last_error("inverse: device ordinal out of range");
        return SCATT_ERR_ARG;
    }
    std::lock_guard<std::mutex> lock(g_attr_mutex);
    const unsigned long long bit = 1ull << dev;
    if (g_attr_done[scheme] & bit) return SCATT_OK;
    const int st = set();
    if (st == SCATT_OK) g_attr_done[scheme] |= bit;
    return st;
}

}  // namespace

int gj_max_order() {
    // shared memory per panel: n * (NB doubles + 2 ints) + reduction scratch
    int lo = 1, hi = 1 << 16;
    while (lo < hi) {
        const int mid = (lo + hi + 1) / 2;
        if (panel_smem_bytes(mid) <= PANEL_SMEM_LIMIT) lo = mid; else hi = mid - 1;
    }
    return lo;
}

int gj_inverse_batched(const GjEntry* entries_dev, int count, int nmax,
                       bool symmetrize, cudaStream_t stream) {
    if (count <= 0 || nmax <= 0) return SCATT_OK;
    if (nmax > gj_max_order()) {
        set_last_error("gj_inverse_batched: order " + std::to_string(nmax) +
                       " exceeds the single-CTA panel limit " + std::to_string(gj_max_order()));
        return SCATT_ERR_SIZE;
    }
    const size_t smem = panel_smem_bytes(nmax);
    SCATT_TRY(once_per_device(0, [&]() -> int {
        SCATT_CUDA_TRY(cudaFuncSetAttribute(gj_update2_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)U2_SMEM));
        SCATT_CUDA_TRY(cudaFuncSetAttribute(gj_panel_kernel,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)PANEL_SMEM_LIMIT));
        return SCATT_OK;
    }));
    const int steps = (nmax + NB - 1) / NB;
    const int tiles = (nmax + UBM - 1) / UBM;
    dim3 ugrid(tiles, tiles, count);
    const size_t smem_reg = 2 * (size_t)nmax * sizeof(int);
    // panel v4: W warps with at most 2 rows of 16 columns per thread
    const int W4 = std::max(1, (nmax + 63) / 64);
    const int T4 = 32 * W4;
    for (int kb = 0; kb < steps; ++kb) {
        if (nmax <= 512) {
            gj_panel5_kernel<2, 256><<<count, T4, smem_reg, stream>>>(entries_dev, kb);
        } else if (nmax <= 1280) {
            gj_panel5_kernel<2, 640><<<count, T4, smem_reg, stream>>>(entries_dev, kb);
        } else {
            gj_panel_kernel<<<count, PANEL_THREADS, smem, stream>>>(entries_dev, kb);
        }
        gj_update2_kernel<<<ugrid, U2T, U2_SMEM, stream>>>(entries_dev, kb);
    }
    const int ft = (nmax + FT - 1) / FT;
    gj_finalize_kernel<<<dim3(ft, ft, count), FT * 8, 0, stream>>>(entries_dev, NB, symmetrize ? 1 : 0, 0);
    SCATT_CUDA_TRY(cudaGetLastError());
    SCATT_COUNT_LAUNCH(2 * steps + 1);
    return SCATT_OK;
}

bool inverse_tune_lookup(int n, int count, InverseTune* out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return false;
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    if (g_tune.empty()) return false;
    const auto it = g_tune.find(std::make_tuple(dev, n, count));
    if (it == g_tune.end()) return false;
    *out = it->second;
    return true;
}

void inverse_tune_store(int device, int n, int count, const InverseTune& t) {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    g_tune[std::make_tuple(device, n, count)] = t;
}

int gj_inverse_batched2(const GjEntry* entries_dev, int count, int nmax, bool symmetrize,
                        cudaStream_t stream, int force_pcfg) {
    if (count <= 0 || nmax <= 0) return SCATT_OK;
    if (nmax > 1280) return gj_inverse_batched(entries_dev, count, nmax, symmetrize, stream);
    if (force_pcfg >= GJ_PANEL_SHAPES) {
        set_last_error("inverse: the cluster panels run on the row-contiguous scheme only");
        return SCATT_ERR_ARG;
    }
    SCATT_TRY(once_per_device(1, [&]() -> int {
        SCATT_CUDA_TRY(cudaFuncSetAttribute(gj2_narrow_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)U2_SMEM));
        return SCATT_OK;
    }));
    const int outer = (nmax + OB - 1) / OB;
    const int tiles = (nmax + 63) / 64;
    int pcfg, pt;
    SCATT_TRY(panel_shape(nmax, pcfg, pt, force_pcfg));
    const size_t lab_smem = 2 * (size_t)nmax * sizeof(int);
    int launches = 0;
    for (int K = 0; K < outer; ++K) {
        for (int sub = 0; sub < OB / NB; ++sub) {
            SCATT_TRY((launch_panel<false, OB>(pcfg, count, pt, lab_smem, stream, entries_dev, K, sub, 0)));
            gj2_narrow_kernel<<<dim3(tiles, 1, count), U2T, U2_SMEM, stream>>>(entries_dev, K, sub);
            launches += 2;
        }
        gj2_trail2_kernel<<<dim3(tiles, tiles, count), U2T, 0, stream>>>(entries_dev, K);
        ++launches;
    }
    const int ft = (nmax + FT - 1) / FT;
    gj_finalize_kernel<<<dim3(ft, ft, count), FT * 8, 0, stream>>>(entries_dev, OB, symmetrize ? 1 : 0, 0);
    SCATT_CUDA_TRY(cudaGetLastError());
    SCATT_COUNT_LAUNCH(launches + 1);
    return SCATT_OK;
}

namespace {

// The row-contiguous two-level inverse with W-column windows.
template <int W>
int batched3_window(const GjEntry* entries_dev, int count, int nmax, bool symmetrize, cudaStream_t stream,
                    bool look_ahead, int force_pcfg) {
    const int outer = (nmax + W - 1) / W;
    const int tiles = (nmax + 63) / 64;
    const int mtiles = (nmax + T3M - 1) / T3M;
    constexpr int WT = W / 64;                   // 64-column tiles per window
    int pcfg, pt;
    SCATT_TRY(panel_shape(nmax, pcfg, pt, force_pcfg));
    const size_t lab_smem = 2 * (size_t)nmax * sizeof(int);
    int launches = 0;
    auto chain = [&](int K, cudaStream_t st, int la) -> int {
        for (int sub = 0; sub < W / NB; ++sub) {
            SCATT_TRY((launch_panel<true, W>(pcfg, count, pt, lab_smem, st, entries_dev, K, sub, la, nmax)));
            gj3_narrow_kernel<W><<<dim3(tiles, WT, count), U2T, NARROW3_SMEM, st>>>(entries_dev, K, sub, la);
            launches += 2;
        }
        return SCATT_OK;
    };
    // trailing update of window K over column tiles [lo, lo + cnt), skipping [skip_lo, skip_lo + skip_n)
    auto trail = [&](int K, int la, int lo, int cnt, int skip_lo, int skip_n, cudaStream_t st) {
        if (cnt <= 0) return;
        if (W == 64) {
            // -1: every column tile; t >= 0: only tile t; -2 - t: every tile but t
            const int cols = skip_n > 0 ? -2 - skip_lo : (cnt == tiles ? -1 : lo);
            gj3_trail_kernel<<<dim3(mtiles, cnt, count), U2T, TRAIL3_SMEM, st>>>(entries_dev, K, la, cols);
        } else {
            gj3_trail128_kernel<<<dim3(mtiles, cnt, count), U2T, TRAIL128_SMEM, st>>>(entries_dev, K, la, lo,
                                                                                    skip_lo, skip_n);
        }
        ++launches;
    };
    if (!look_ahead || outer < 2) {
        for (int K = 0; K < outer; ++K) {
            SCATT_TRY(chain(K, stream, 0));
            trail(K, 0, 0, tiles, 0, 0, stream);
        }
    } else {
        std::lock_guard<std::mutex> lock(g_la_mutex);
        LookAhead* la = nullptr;
        SCATT_TRY(look_ahead_resources(stream, &la));
        SCATT_TRY(chain(0, stream, 1));
        for (int K = 0; K < outer; ++K) {
            if (K + 1 < outer) {
                // the next window's column tiles first, then its chain beside the rest of the update
                const int nlo = (K + 1) * WT, ncnt = std::min(WT, tiles - nlo);
                trail(K, 1, nlo, ncnt, 0, 0, stream);
                SCATT_CUDA_TRY(cudaEventRecord(la->ev_main, stream));
                SCATT_CUDA_TRY(cudaStreamWaitEvent(la->side, la->ev_main, 0));
                SCATT_TRY(chain(K + 1, la->side, 1));
                SCATT_CUDA_TRY(cudaEventRecord(la->ev_side, la->side));
                trail(K, 1, 0, tiles - ncnt, nlo, ncnt, stream);
                SCATT_CUDA_TRY(cudaStreamWaitEvent(stream, la->ev_side, 0));
            } else {
                trail(K, 1, 0, tiles, 0, 0, stream);
            }
        }
    }
    const int ft = (nmax + FT - 1) / FT;
    gj_finalize_kernel<<<dim3(ft, ft, count), FT * 8, 0, stream>>>(entries_dev, W, symmetrize ? 1 : 0, 1);
    SCATT_CUDA_TRY(cudaGetLastError());
    SCATT_COUNT_LAUNCH(launches + 1);
    return SCATT_OK;
}

}  // namespace

int gj_inverse_batched3(const GjEntry* entries_dev, int count, int nmax, bool symmetrize,
                        cudaStream_t stream, bool look_ahead, int force_pcfg, int window) {
    if (count <= 0 || nmax <= 0) return SCATT_OK;
    if (window != 64 && window != 128) {
        set_last_error("inverse: window width must be 64 or 128, got " + std::to_string(window));
        return SCATT_ERR_ARG;
    }
    SCATT_TRY(once_per_device(2, [&]() -> int {
        SCATT_CUDA_TRY(cudaFuncSetAttribute(gj3_narrow_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)NARROW3_SMEM));
        SCATT_CUDA_TRY(cudaFuncSetAttribute(gj3_narrow_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)NARROW3_SMEM));
        SCATT_CUDA_TRY(cudaFuncSetAttribute(gj3_trail_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)TRAIL3_SMEM));
        SCATT_CUDA_TRY(cudaFuncSetAttribute(gj3_trail128_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)TRAIL128_SMEM));
        return SCATT_OK;
    }));
    return window == 128 ? batched3_window<128>(entries_dev, count, nmax, symmetrize, stream, look_ahead, force_pcfg)
                         : batched3_window<64>(entries_dev, count, nmax, symmetrize, stream, look_ahead, force_pcfg);
}

}  // namespace scatt
