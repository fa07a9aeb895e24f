// capi.cu -- extern "C" entry points: error handling, angular algebra,
// device building blocks.  The per-energy-batch solver entry points live in
// solver.cu.
#include <cstring>
#include <string>
#include <vector>

#include "angular.hpp"
#include "common.cuh"
#include "devbuf.cuh"
#include "riccati.cuh"

namespace scatt {

namespace {
thread_local std::string g_last_error;
}
// scheme of every dense inverse (see gj_inverse_selected)
std::atomic<int> g_inverse_scheme{0};

void set_last_error(const std::string& msg) { g_last_error = msg; }

std::atomic<unsigned long long>& launch_counter() {
    static std::atomic<unsigned long long> c{0};
    return c;
}

int require_device() {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        (void)cudaGetLastError();
        set_last_error("no CUDA device visible (the library has no CPU fallback)");
        return SCATT_ERR_NO_DEVICE;
    }
    return SCATT_OK;
}

__global__ void fill_test_matrices(double* A, int n, int count, unsigned seed) {
    const size_t total = (size_t)n * n * count;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total;
         idx += (size_t)gridDim.x * blockDim.x) {
        unsigned h = (unsigned)(idx * 2654435761u) ^ seed;
        h ^= h >> 13; h *= 0x5bd1e995u; h ^= h >> 15;
        const size_t within = idx % ((size_t)n * n);
        const int i = (int)(within % n), j = (int)(within / n);
        A[idx] = (double)(h & 0xffffff) / 16777216.0 - 0.5 + (i == j ? 2.0 : 0.0);
    }
}

}  // namespace scatt

using namespace scatt;

namespace {

// Seeded test matrices (uniform entries in [-0.5, 0.5) plus 2 on the
// diagonal) and their inverse entries (panel windows sized for the
// look-ahead), for timing the inverse's kernels alone.
struct InverseBench {
    int n = 0, count = 0;
    DevBuf<double> dA, dW, dO, dS, dP;
    DevBuf<int> dsig, drid, dst, dsg;
    DevBuf<GjEntry> dent;

    int setup(int n_, int count_) {
        n = n_;
        count = count_;
        const size_t nn = (size_t)n * n;
        SCATT_TRY(dP.alloc((size_t)4 * n * GJ_WINDOW_MAX * count));
        SCATT_TRY(dsg.alloc((size_t)4 * n * count));
        SCATT_TRY(dA.alloc(nn * count));
        SCATT_TRY(dS.alloc(nn * count));
        SCATT_TRY(dW.alloc(nn * count));
        SCATT_TRY(dO.alloc(nn * count));
        SCATT_TRY(dsig.alloc((size_t)n * count));
        SCATT_TRY(drid.alloc((size_t)n * count));
        SCATT_TRY(dst.alloc(2 * (size_t)count));
        fill_test_matrices<<<1024, 256>>>(dS.p, n, count, 12345u);
        SCATT_CUDA_TRY(cudaGetLastError());
        std::vector<GjEntry> ent(count);
        for (int b = 0; b < count; ++b)
            ent[b] = GjEntry{dA.p + nn * b, dW.p + nn * b, dO.p + nn * b, dsig.p + (size_t)n * b,
                             drid.p + (size_t)n * b, dst.p + 2 * b, n, n, n,
                             dP.p + (size_t)4 * n * GJ_WINDOW_MAX * b, dsg.p + (size_t)4 * n * b};
        return dent.upload(ent);
    }

    // mean milliseconds of run() over reps calls after one untimed call; the
    // input is restored before each call, outside the timed span
    template <class F>
    int time(int reps, double* ms_out, F run) {
        const size_t bytes = (size_t)n * n * count * sizeof(double);
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        SCATT_CUDA_TRY(cudaEventCreate(&e0));
        if (cudaEventCreate(&e1) != cudaSuccess) {
            cudaEventDestroy(e0);
            return cuda_status(cudaErrorMemoryAllocation, "cudaEventCreate");
        }
        double total = 0.0;
        int st = SCATT_OK;
        for (int r = 0; r < reps + 1 && st == SCATT_OK; ++r) {
            cudaError_t ce = cudaMemcpyAsync(dA.p, dS.p, bytes, cudaMemcpyDeviceToDevice, 0);
            if (ce == cudaSuccess) ce = cudaEventRecord(e0, 0);
            if (ce != cudaSuccess) { st = cuda_status(ce, "inverse timing"); break; }
            st = run();
            if (st != SCATT_OK) break;
            ce = cudaEventRecord(e1, 0);
            if (ce == cudaSuccess) ce = cudaEventSynchronize(e1);
            float ms = 0.f;
            if (ce == cudaSuccess) ce = cudaEventElapsedTime(&ms, e0, e1);
            if (ce != cudaSuccess) { st = cuda_status(ce, "inverse timing"); break; }
            if (r > 0) total += ms;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (st == SCATT_OK) *ms_out = total / reps;
        return st;
    }
};

}  // namespace

extern "C" {

const char* scatt_version(void) { return "spion-emol_b200 0.1 (sm_100a, FP64 DMMA)"; }

const char* scatt_last_error(void) { return g_last_error.c_str(); }

int scatt_device_count(int* count) {
    if (!count) return SCATT_ERR_ARG;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        (void)cudaGetLastError();
        n = 0;
    }
    *count = n;
    return SCATT_OK;
}

double scatt_wigner3j(int j1, int j2, int j3, int m1, int m2, int m3) {
    return wigner3j(j1, j2, j3, m1, m2, m3);
}
double scatt_gaunt_real(int l1, int m1, int l2, int m2, int l3, int m3) {
    return gaunt_real(l1, m1, l2, m2, l3, m3);
}
double scatt_angular_dipole(int l_mu, int m_mu, int q, int l_nu, int m_nu) {
    return angular_dipole(l_mu, m_mu, q, l_nu, m_nu);
}
double scatt_velocity_coef(int l_mu, int l_nu) { return velocity_coef(l_mu, l_nu); }
double scatt_riccati_j(int l, double x) { return scatt::riccati_j(l, x); }
double scatt_riccati_y(int l, double x) { return scatt::riccati_y(l, x); }

int scatt_inverse_batched(int n, int count, const double* A, double* out, int symmetrize,
                          int* status) {
    if (n <= 0 || count <= 0 || !A || !out) {
        set_last_error("scatt_inverse_batched: bad arguments");
        return SCATT_ERR_ARG;
    }
    SCATT_TRY(require_device());
    const size_t nn = (size_t)n * n;
    DevBuf<double> dA, dW, dO, dP;
    DevBuf<int> dsig, drid, dst, dsg;
    SCATT_TRY(dA.alloc(nn * count));
    SCATT_TRY(dW.alloc(nn * count));
    SCATT_TRY(dO.alloc(nn * count));
    SCATT_TRY(dP.alloc((size_t)4 * n * GJ_WINDOW_MAX * count));
    SCATT_TRY(dsig.alloc((size_t)n * count));
    SCATT_TRY(drid.alloc((size_t)n * count));
    SCATT_TRY(dsg.alloc((size_t)4 * n * count));
    SCATT_TRY(dst.alloc(2 * (size_t)count));
    SCATT_CUDA_TRY(cudaMemcpy(dA.p, A, nn * count * sizeof(double), cudaMemcpyHostToDevice));
    SCATT_CUDA_TRY(cudaMemset(dst.p, 0, 2 * count * sizeof(int)));
    std::vector<GjEntry> ent(count);
    for (int b = 0; b < count; ++b) {
        ent[b] = GjEntry{dA.p + nn * b, dW.p + nn * b, dO.p + nn * b, dsig.p + (size_t)n * b,
                         drid.p + (size_t)n * b, dst.p + 2 * b, n, n, n,
                         dP.p + (size_t)4 * n * GJ_WINDOW_MAX * b, dsg.p + (size_t)4 * n * b};
    }
    DevBuf<GjEntry> dent;
    SCATT_TRY(dent.upload(ent));
    SCATT_TRY(gj_inverse_selected(dent.p, count, n, symmetrize != 0, 0, true));
    SCATT_CUDA_TRY(cudaDeviceSynchronize());
    SCATT_CUDA_TRY(cudaMemcpy(out, dO.p, nn * count * sizeof(double), cudaMemcpyDeviceToHost));
    std::vector<int> st(2 * count);
    SCATT_CUDA_TRY(cudaMemcpy(st.data(), dst.p, st.size() * sizeof(int), cudaMemcpyDeviceToHost));
    if (status) std::memcpy(status, st.data(), st.size() * sizeof(int));
    for (int b = 0; b < count; ++b) {
        if (st[2 * b] == DEV_SINGULAR) {
            set_last_error("scatt_inverse_batched: singular pivot in matrix " + std::to_string(b) +
                           " at column " + std::to_string(st[2 * b + 1]));
            return SCATT_ERR_SINGULAR;
        }
        if (st[2 * b] == DEV_NONFINITE) {
            set_last_error("scatt_inverse_batched: non-finite pivot in matrix " + std::to_string(b) +
                           " at column " + std::to_string(st[2 * b + 1]));
            return SCATT_ERR_NONFINITE;
        }
    }
    return SCATT_OK;
}

int scatt_dgemm(int opA, int opB, int M, int N, int K, double alpha, const double* A, int lda,
                const double* B, int ldb, double beta, double* C, int ldc) {
    if (M <= 0 || N <= 0 || K < 0 || !A || !B || !C) {
        set_last_error("scatt_dgemm: bad arguments");
        return SCATT_ERR_ARG;
    }
    SCATT_TRY(require_device());
    const size_t sa = (size_t)lda * (opA ? M : K), sb = (size_t)ldb * (opB ? K : N);
    const size_t sc = (size_t)ldc * N;
    DevBuf<double> dA, dB, dC;
    SCATT_TRY(dA.alloc(sa ? sa : 1));
    SCATT_TRY(dB.alloc(sb ? sb : 1));
    SCATT_TRY(dC.alloc(sc));
    SCATT_CUDA_TRY(cudaMemcpy(dA.p, A, sa * sizeof(double), cudaMemcpyHostToDevice));
    SCATT_CUDA_TRY(cudaMemcpy(dB.p, B, sb * sizeof(double), cudaMemcpyHostToDevice));
    SCATT_CUDA_TRY(cudaMemcpy(dC.p, C, sc * sizeof(double), cudaMemcpyHostToDevice));
    GemmEntry e{dA.p, dB.p, dC.p, M, N, K, lda, ldb, ldc, alpha, beta};
    DevBuf<GemmEntry> de;
    SCATT_TRY(de.upload(std::vector<GemmEntry>{e}));
    SCATT_TRY(gemm_batched(de.p, 1, M, N, opA, opB, 0));
    SCATT_CUDA_TRY(cudaDeviceSynchronize());
    SCATT_CUDA_TRY(cudaMemcpy(C, dC.p, sc * sizeof(double), cudaMemcpyDeviceToHost));
    return SCATT_OK;
}

int scatt_bench_gemm(int opA, int opB, int M, int N, int K, int count, int sym, int reps, double* ms_per_call) {
    if (M <= 0 || N <= 0 || K <= 0 || count <= 0 || reps <= 0 || !ms_per_call || (sym && M != N) ||
        opA < 0 || opA > 1 || opB < 0 || opB > 1) {
        set_last_error("scatt_bench_gemm: bad arguments");
        return SCATT_ERR_ARG;
    }
    SCATT_TRY(require_device());
    const size_t sa = (size_t)M * K, sb = (size_t)K * N, sc = (size_t)M * N;
    DevBuf<double> dA, dB, dC;
    SCATT_TRY(dA.alloc(sa * count));
    SCATT_TRY(dB.alloc(sb * count));
    SCATT_TRY(dC.alloc(sc * count));
    fill_test_matrices<<<1024, 256>>>(dA.p, 1, (int)std::min<size_t>(sa * count, 1u << 30), 7u);
    fill_test_matrices<<<1024, 256>>>(dB.p, 1, (int)std::min<size_t>(sb * count, 1u << 30), 11u);
    SCATT_CUDA_TRY(cudaMemset(dC.p, 0, sc * count * sizeof(double)));
    std::vector<GemmEntry> ent(count);
    for (int b = 0; b < count; ++b)
        ent[b] = GemmEntry{dA.p + sa * b, dB.p + sb * b, dC.p + sc * b, M, N, K,
                           opA ? K : M, opB ? N : K, M, 1.0, 0.0, sym ? 1 : 0};
    DevBuf<GemmEntry> de;
    SCATT_TRY(de.upload(ent));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    SCATT_CUDA_TRY(cudaEventCreate(&e0));
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return cuda_status(cudaErrorMemoryAllocation, "cudaEventCreate");
    }
    double total = 0.0;
    int st = SCATT_OK;
    for (int r = 0; r < reps + 1 && st == SCATT_OK; ++r) {
        cudaError_t ce = cudaEventRecord(e0, 0);
        if (ce != cudaSuccess) { st = cuda_status(ce, "gemm timing"); break; }
        st = gemm_batched(de.p, count, M, N, opA, opB, 0);
        if (st != SCATT_OK) break;
        ce = cudaEventRecord(e1, 0);
        if (ce == cudaSuccess) ce = cudaEventSynchronize(e1);
        float ms = 0.f;
        if (ce == cudaSuccess) ce = cudaEventElapsedTime(&ms, e0, e1);
        if (ce != cudaSuccess) { st = cuda_status(ce, "gemm timing"); break; }
        if (r > 0) total += ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st == SCATT_OK) *ms_per_call = total / reps;
    return st;
}

int scatt_set_inverse_blocking(int scheme) {
    if (scheme < 0 || scheme > 6) {
        set_last_error("scatt_set_inverse_blocking: scheme must be in 0..6");
        return SCATT_ERR_ARG;
    }
    g_inverse_scheme.store(scheme, std::memory_order_relaxed);
    return SCATT_OK;
}

int scatt_bench_inverse(int n, int count, int reps, double* ms_per_call) {
    if (n <= 0 || count <= 0 || reps <= 0 || !ms_per_call) return SCATT_ERR_ARG;
    SCATT_TRY(require_device());
    InverseBench bench;
    SCATT_TRY(bench.setup(n, count));
    return bench.time(reps, ms_per_call, [&]() { return gj_inverse_selected(bench.dent.p, count, n, true, 0, true); });
}

int scatt_autotune_inverse(int n, int count, int reps, int* scheme, int* panel, int* look_ahead, int* window,
                           double* best_ms) {
    if (n <= 0 || n > 8192 || count <= 0 || reps <= 0) {
        set_last_error("scatt_autotune_inverse: order must be in [1, 8192], batch and reps positive");
        return SCATT_ERR_ARG;
    }
    SCATT_TRY(require_device());
    int dev = 0;
    SCATT_CUDA_TRY(cudaGetDevice(&dev));
    InverseBench bench;
    SCATT_TRY(bench.setup(n, count));
    InverseTune best;
    double best_t = 1e300;
    // above one CTA's panel (1280 rows) only the row-contiguous scheme with the cluster panel runs
    const bool cluster = n > gj_panel_capacity(GJ_PANEL_SHAPES - 1);
    for (int sch = cluster ? 3 : 2; sch <= 3; ++sch)
        for (int p = 0; p <= GJ_PANEL_SMALL_CLUSTER; ++p) {
            if (p == GJ_PANEL_SMALL_CLUSTER) {
                if (sch != 3 || n > 3072) continue;       // the small cluster panel: row-contiguous only
            } else if (cluster ? p != GJ_PANEL_SHAPES : (p == GJ_PANEL_SHAPES || n > gj_panel_capacity(p))) {
                continue;
            }
            for (int la = 0; la <= (sch == 3 ? 1 : 0); ++la)
                for (int w = 64; w <= (sch == 3 ? GJ_WINDOW_MAX : 64); w *= 2) {
                    double ms = 0.0;
                    SCATT_TRY(bench.time(reps, &ms, [&]() {
                        return sch == 3 ? gj_inverse_batched3(bench.dent.p, count, n, true, 0, la != 0, p, w)
                                        : gj_inverse_batched2(bench.dent.p, count, n, true, 0, p);
                    }));
                    if (ms < best_t) {
                        best_t = ms;
                        best.scheme = sch;
                        best.pcfg = p;
                        best.look_ahead = la;
                        best.window = w;
                    }
                }
        }
    inverse_tune_store(dev, n, count, best);
    if (scheme) *scheme = best.scheme;
    if (panel) *panel = best.pcfg;
    if (look_ahead) *look_ahead = best.look_ahead;
    if (window) *window = best.window;
    if (best_ms) *best_ms = best_t;
    return SCATT_OK;
}

}  // extern "C"
