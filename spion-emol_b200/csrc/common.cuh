// common.cuh -- shared definitions for the sm_100a scattering library.
//
// All matrices are FP64, column-major (element (i, j) at p[i + j * ld]),
// matching the Eigen default layout the reference interfaces use.
#pragma once

#include <cuda_runtime.h>
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <string>

#include "scatt_b200.h"

namespace scatt {

// Error bookkeeping: every host entry point returns an int status; the last
// error message is kept per thread (see capi.cu).
void set_last_error(const std::string& msg);
// SCATT_ERR_NO_DEVICE (with the last error set) when no CUDA device is visible.
int require_device();

#define SCATT_CUDA_TRY(expr)                                                    \
    do {                                                                        \
        cudaError_t _e = (expr);                                                \
        if (_e != cudaSuccess) {                                                \
            ::scatt::set_last_error(std::string(#expr) + ": " +                 \
                                    cudaGetErrorString(_e));                    \
            return SCATT_ERR_CUDA;                                              \
        }                                                                       \
    } while (0)

inline int cuda_status(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        set_last_error(std::string(what) + ": " + cudaGetErrorString(e));
        return SCATT_ERR_CUDA;
    }
    return SCATT_OK;
}
#define SCATT_CUDA_TRY_RET(expr) ::scatt::cuda_status((expr), #expr)

#define SCATT_TRY(expr)                                                         \
    do {                                                                        \
        int _s = (expr);                                                        \
        if (_s != SCATT_OK) return _s;                                          \
    } while (0)

// Kernel launches issued by the library since load, by every thread
// (benchmark bookkeeping; atomic because solves may run on several threads).
std::atomic<unsigned long long>& launch_counter();
#define SCATT_COUNT_LAUNCH(n) (::scatt::launch_counter().fetch_add((n), std::memory_order_relaxed))

// Device-side status codes written into per-matrix status words.
enum DeviceStatus : int {
    DEV_OK = 0,
    DEV_SINGULAR = 1,      // zero pivot encountered
    DEV_NONFINITE = 2,     // NaN / Inf pivot
};

// ---------------------------------------------------------------- GEMM
// One entry of a batched GEMM:  C = alpha * op(A) * op(B) + beta * C.
// op(A) is M x K, op(B) is K x N.  Entries with M, N or K <= 0 are skipped
// (K <= 0 with beta != 1 still scales C).
struct GemmEntry {
    const double* A;
    const double* B;
    double*       C;
    int M, N, K;
    int lda, ldb, ldc;
    double alpha, beta;
    // 1: op(A) op(B) is symmetric (M == N) and C starts symmetric: only the
    // lower-triangle tiles are computed and each result is mirrored, so C
    // comes out exactly symmetric
    int sym = 0;
};

// opA / opB: 0 = no transpose, 1 = transpose.  `entries` is a DEVICE array.
int gemm_batched(const GemmEntry* entries_dev, int count, int maxM, int maxN,
                 int opA, int opB, cudaStream_t stream);

// ---------------------------------------------------------------- GJ inverse
// Batched in-place Gauss-Jordan inversion with partial (row) pivoting,
// blocked by GJ_NB columns.  Each matrix has its own order n (<= nmax).
struct GjEntry {
    double* A;        // input matrix (n x n, ld), destroyed
    double* W;        // workspace of the same shape (ping-pong buffer)
    double* out;      // output (n x n, ldo): inverse (optionally symmetrised)
    int*    sigma;    // n ints: row map of the current block step
    int*    rowid;    // n ints: original row index at each position
    int*    status;   // 1 int: DeviceStatus (first failing column in status[1])
    int n, ld, ldo;
    double* P = nullptr;   // optional panel-window buffers, 2 x (ld x window) (4 x with look-ahead)
    int*    sigt = nullptr; // optional composite row maps of the 64-column window (2 n, 4 n with look-ahead)
};

constexpr int GJ_NB = 16;

// Largest n the single-CTA panel factorisation holds in shared memory.
int gj_max_order();

// Runs the whole inversion (ceil(nmax / GJ_NB) block steps).  `entries_dev`
// is a DEVICE array; `symmetrize` writes 0.5 * (X + X^T) into `out`.
int gj_inverse_batched(const GjEntry* entries_dev, int count, int nmax,
                       bool symmetrize, cudaStream_t stream);

// Two-level blocked variant (64-column windows, rank-64 trailing updates) for
// n <= 1280; every entry must carry P (2 x ld x 64 doubles) and sigt (2 n ints).
// pcfg >= 0 forces the panel shape (see gj_panel_capacity).
int gj_inverse_batched2(const GjEntry* entries_dev, int count, int nmax,
                        bool symmetrize, cudaStream_t stream, int pcfg = -1);

// Two-level variant on the row-contiguous view: the column-major buffer of A
// is treated as the row-major B = A^T (inv(A) = inv(B)^T), so pivot rows and
// window rows are contiguous runs.  Pivoting is partial pivoting on B, i.e.
// by columns of A; for symmetric A it is the row-pivoting sequence of A.
// `window` (64 or 128) is the width of the outer step: a 128-column window
// halves the trailing updates' C-tile traffic per flop.  With look_ahead the
// 16-column panels of the next window run on a high-priority side stream
// beside the trailing update of the current one; then every entry needs P of
// 4 x ld x window doubles and sigt of 4 n ints (without it, 2 x ld x window
// and 2 n).  Orders above 1280 run the panels on a thread-block cluster.
int gj_inverse_batched3(const GjEntry* entries_dev, int count, int nmax,
                        bool symmetrize, cudaStream_t stream, bool look_ahead, int pcfg = -1,
                        int window = 64);

// Widest window of the two-level inverses; entries carrying P of 4 x ld x
// GJ_WINDOW_MAX doubles fit every choice.
constexpr int GJ_WINDOW_MAX = 128;

// Panel shapes of the two-level inverses, as rows per thread x warps: 1x8,
// 2x8, 3x8, 3x12, 5x8.  Shape p factors panels of up to gj_panel_capacity(p)
// rows; the default is the smallest shape that holds the order.
constexpr int GJ_PANEL_SHAPES = 5;
// Two more panel configurations of the row-contiguous scheme: GJ_PANEL_SHAPES
// itself (a cluster of 1024-row CTAs, orders above 1280) and the small
// cluster panel (384-row CTAs that fit beside the trailing update, any order
// up to 3072).
constexpr int GJ_PANEL_SMALL_CLUSTER = GJ_PANEL_SHAPES + 1;
inline int gj_panel_capacity(int pcfg) {
    constexpr int cap[GJ_PANEL_SHAPES] = {256, 512, 768, 1152, 1280};
    return cap[pcfg];
}

// A measured choice of scheme (2 or 3), panel shape, look-ahead and window
// width for one (device, order, batch).  The autotuner
// (scatt_autotune_inverse) stores them; the automatic scheme uses a stored
// choice for an exact match of the current device, order and batch, and its
// fixed rule otherwise.
struct InverseTune {
    int scheme = 0, pcfg = -1, look_ahead = 1, window = 64;
};
bool inverse_tune_lookup(int n, int count, InverseTune* out);
void inverse_tune_store(int device, int n, int count, const InverseTune& t);

// Scheme of every dense inverse (entry points and solver): 0 = automatic
// (row-contiguous two-level above order 512, where its contiguous pivot-row
// tiles pay; column-major two-level below), 1 = single-level,
// 2 = column-major two-level, 3 = row-contiguous two-level, 4 = scheme 3
// with 128-column windows (where the entries' buffers hold them), 5 / 6 =
// schemes 3 / 4 with the small cluster panel.  Process-wide;
// atomic because it may be set while another thread solves (a call reads it
// once per inverse, so a change applies from the next inverse on).
extern std::atomic<int> g_inverse_scheme;

// The scheme selected by g_inverse_scheme (entries must carry P and sigt).
// look_ahead: as for gj_inverse_batched3 (entries sized for it); wcap: the
// widest window the entries' P holds (64 or GJ_WINDOW_MAX).
inline int gj_inverse_selected(const GjEntry* entries_dev, int count, int nmax,
                               bool symmetrize, cudaStream_t stream, bool look_ahead,
                               int wcap = GJ_WINDOW_MAX) {
    switch (g_inverse_scheme.load(std::memory_order_relaxed)) {
        case 1: return gj_inverse_batched(entries_dev, count, nmax, symmetrize, stream);
        case 2: return gj_inverse_batched2(entries_dev, count, nmax, symmetrize, stream);
        case 3: return gj_inverse_batched3(entries_dev, count, nmax, symmetrize, stream, look_ahead);
        case 4: return gj_inverse_batched3(entries_dev, count, nmax, symmetrize, stream, look_ahead, -1,
                                           wcap >= 128 ? 128 : 64);
        case 5: return gj_inverse_batched3(entries_dev, count, nmax, symmetrize, stream, look_ahead,
                                           GJ_PANEL_SMALL_CLUSTER, 64);
        case 6: return gj_inverse_batched3(entries_dev, count, nmax, symmetrize, stream, look_ahead,
                                           GJ_PANEL_SMALL_CLUSTER, wcap >= 128 ? 128 : 64);
        default: {
            InverseTune t;
            if (inverse_tune_lookup(nmax, count, &t)) {
                if (t.scheme == 3)
                    return gj_inverse_batched3(entries_dev, count, nmax, symmetrize, stream,
                                               look_ahead && t.look_ahead, t.pcfg,
                                               t.window <= wcap ? t.window : 64);
                return gj_inverse_batched2(entries_dev, count, nmax, symmetrize, stream, t.pcfg);
            }
            return nmax > 512 ? gj_inverse_batched3(entries_dev, count, nmax, symmetrize, stream, look_ahead)
                              : gj_inverse_batched2(entries_dev, count, nmax, symmetrize, stream);
        }
    }
}

}  // namespace scatt
