// hartree.cu -- the Hartree potential of the preprocessing step from the
// density's single-centre multipoles, by the radial Poisson integrals
// (preprocessing/src/potential/Hartree.hpp:71-246, build_V_H):
//
//   V_lm(r) = 4 pi / (2l + 1) [ r^-(l+1) int_0^r rho_lm r'^(l+2) dr'
//                             + r^l      int_r^R rho_lm r'^(1-l) dr' ]
//
// on the uniform grid r_k = r0 + k dr, with the cumulative integrator of
// preprocessing/src/sce/RadialGrid.hpp:84-100 (I_0 = 0, I_k+1 = I_k +
// h/12 (5 f_k + 8 f_k+1 - f_k+2), the last interval by the mirrored
// stencil) and the reference's guards: channels above the overflow-safe l
// and channels whose |rho_lm| stays below 1e-12 are 0, a non-finite value
// is 0, at r = 0 the first term is 0 and f_out = 0 for l >= 1, and
// V_00(0) = 4 pi int_0^R rho_00 r' dr'.
//
// One CTA per channel.  The two running integrals are block-wide prefix
// sums: each thread owns a contiguous run of the row's intervals, sums it,
// the CTA scans the thread sums with warp shuffles, and each thread then
// walks its run again from its offset, writing V.  A point costs a few
// FP64 pow() evaluations per pass (the integrands' r^(l+2), r^(1-l)), so
// the step is bound by the FP64 pipe rather than by the 8 bytes it reads
// and the 8 it writes per point; it runs once per molecule.
#include <algorithm>
#include <cmath>
#include <string>

#include "common.cuh"
#include "devbuf.cuh"

namespace scatt {
namespace {

constexpr int HT_THREADS = 256;

struct Pair {
    double a, b;
};

__device__ __forceinline__ double pw(double r, int e) { return pow(r, (double)e); }

// the two integrands at point k of a row
__device__ __forceinline__ Pair integrands(const double* rho, int k, int l, double r0, double dr) {
    const double r = r0 + k * dr;
    const double x = rho[k];
    Pair f;
    f.a = x * pw(r, l + 2);
    f.b = (l == 0) ? x * r : (r <= 0.0 ? 0.0 : x * pw(r, 1 - l));
    return f;
}

// interval j (from point j to j + 1) of the cumulative integrator, n points
__device__ __forceinline__ Pair increment(const double* rho, int j, int n, int l, double r0, double dr) {
    const double h12 = dr / 12.0;
    Pair s;
    if (j < n - 2) {
        const Pair f0 = integrands(rho, j, l, r0, dr), f1 = integrands(rho, j + 1, l, r0, dr),
                   f2 = integrands(rho, j + 2, l, r0, dr);
        s.a = h12 * (5.0 * f0.a + 8.0 * f1.a - f2.a);
        s.b = h12 * (5.0 * f0.b + 8.0 * f1.b - f2.b);
    } else {
        const Pair f0 = integrands(rho, n - 3, l, r0, dr), f1 = integrands(rho, n - 2, l, r0, dr),
                   f2 = integrands(rho, n - 1, l, r0, dr);
        s.a = h12 * (-f0.a + 8.0 * f1.a + 5.0 * f2.a);
        s.b = h12 * (-f0.b + 8.0 * f1.b + 5.0 * f2.b);
    }
    return s;
}

__device__ __forceinline__ double block_max(double v, double* sh) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    double m = 0.0;
    for (int w = 0; w < HT_THREADS / 32; ++w) m = fmax(m, sh[w]);
    __syncthreads();
    return m;
}

// exclusive prefix of (a, b) over the CTA's threads in order; *tot = the totals
__device__ __forceinline__ Pair block_exclusive_scan(Pair v, Pair* sh, Pair* tot) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    Pair inc = v;
    for (int o = 1; o < 32; o <<= 1) {
        const double ya = __shfl_up_sync(0xffffffffu, inc.a, o), yb = __shfl_up_sync(0xffffffffu, inc.b, o);
        if (lane >= o) { inc.a += ya; inc.b += yb; }
    }
    if (lane == 31) sh[warp] = inc;
    __syncthreads();
    Pair base{0.0, 0.0}, all{0.0, 0.0};
    for (int w = 0; w < HT_THREADS / 32; ++w) {
        if (w < warp) { base.a += sh[w].a; base.b += sh[w].b; }
        all.a += sh[w].a;
        all.b += sh[w].b;
    }
    __syncthreads();
    *tot = all;
    return Pair{base.a + inc.a - v.a, base.b + inc.b - v.b};
}

__global__ void __launch_bounds__(HT_THREADS)
k_hartree(const double* __restrict__ rho_lm, int Nr, double r0, double dr, int l_safe, double* __restrict__ V) {
    __shared__ double shm[HT_THREADS / 32];
    __shared__ Pair shp[HT_THREADS / 32];
    const int ch = blockIdx.x;
    const int l = (int)sqrt((double)ch + 0.5);
    const double* rho = rho_lm + (size_t)ch * Nr;
    double* out = V + (size_t)ch * Nr;
    double mx = 0.0;
    for (int k = threadIdx.x; k < Nr; k += HT_THREADS) mx = fmax(mx, fabs(rho[k]));
    mx = block_max(mx, shm);
    if (l > l_safe || mx < 1e-12) {
        for (int k = threadIdx.x; k < Nr; k += HT_THREADS) out[k] = 0.0;
        return;
    }
    const double pref = 4.0 * 3.14159265358979323846 / (2.0 * l + 1.0);
    // this thread's intervals [j0, j1) of the n - 1
    const int nint = Nr - 1;
    const int per = (nint + HT_THREADS - 1) / HT_THREADS;
    const int j0 = min(nint, (int)threadIdx.x * per), j1 = min(nint, j0 + per);
    Pair own{0.0, 0.0};
    for (int j = j0; j < j1; ++j) {
        const Pair s = increment(rho, j, Nr, l, r0, dr);
        own.a += s.a;
        own.b += s.b;
    }
    Pair tot;
    Pair I = block_exclusive_scan(own, shp, &tot);     // I_in, I_out_left at point j0
    auto emit = [&](int k, const Pair& Ik) {
        const double r = r0 + k * dr;
        const double term1 = (r <= 0.0) ? 0.0 : Ik.a / pw(r, l + 1);
        double v = pref * (term1 + pw(r, l) * (tot.b - Ik.b));
        if (!isfinite(v)) v = 0.0;
        if (l == 0 && k == 0) v = pref * tot.b;
        out[k] = v;
    };
    for (int j = j0; j < j1; ++j) {
        emit(j, I);
        const Pair s = increment(rho, j, Nr, l, r0, dr);
        I.a += s.a;
        I.b += s.b;
    }
    if (j1 == nint && j0 < j1) emit(nint, I);          // the last point: the whole integral
}

}  // namespace
}  // namespace scatt

using namespace scatt;

extern "C" int scatt_hartree(int l_max, int n_rows, int Nr, double r0, double dr, const double* rho_lm,
                             double* V_H) {
    const int n_lm = (l_max + 1) * (l_max + 1);
    if (l_max < 0 || Nr < 3 || !(dr > 0.0) || !rho_lm || !V_H) {
        set_last_error("scatt_hartree: need l_max >= 0, Nr >= 3, dr > 0 and the buffers");
        return SCATT_ERR_ARG;
    }
    if (n_rows < n_lm) {
        set_last_error("build_V_H: rho_lm rows < (Lmax+1)^2");
        return SCATT_ERR_ARG;
    }
    SCATT_TRY(require_device());
    // the largest l whose r^l and r^(1-l) stay finite on the grid (Hartree.hpp:84-110)
    int l_safe = l_max;
    const double r_max = r0 + (Nr - 1) * dr;
    double r_min_pos = 0.0;
    for (int k = 0; k < Nr; ++k)
        if (r0 + k * dr > 0.0) { r_min_pos = r0 + k * dr; break; }
    if (r_max > 1.0) l_safe = std::min(l_safe, (int)(690.0 / std::log(r_max)));
    if (r_min_pos > 0.0 && r_min_pos < 1.0) l_safe = std::min(l_safe, 1 + (int)(690.0 / std::log(1.0 / r_min_pos)));
    cudaStream_t s = nullptr;
    SCATT_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    struct StreamOwner {
        cudaStream_t s;
        ~StreamOwner() { cudaStreamDestroy(s); }
    } own{s};
    const size_t cnt = (size_t)n_lm * Nr;
    DevBuf<double> drho, dV;
    SCATT_TRY(drho.alloc(cnt));
    SCATT_TRY(dV.alloc(cnt));
    SCATT_CUDA_TRY(cudaMemcpyAsync(drho.p, rho_lm, cnt * sizeof(double), cudaMemcpyHostToDevice, s));
    k_hartree<<<n_lm, HT_THREADS, 0, s>>>(drho.p, Nr, r0, dr, l_safe, dV.p);
    SCATT_CUDA_TRY(cudaGetLastError());
    SCATT_COUNT_LAUNCH(1);
    SCATT_CUDA_TRY(cudaMemcpyAsync(V_H, dV.p, cnt * sizeof(double), cudaMemcpyDeviceToHost, s));
    SCATT_CUDA_TRY(cudaStreamSynchronize(s));
    return SCATT_OK;
}
