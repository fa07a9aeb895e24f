// noalloc.cu -- scatt_inverse_batched_noalloc: the batched Gauss-Jordan
// inverse with every device buffer carved from one file-scope scratch array,
// so a call performs no device allocation.  It serves callers that cannot
// call cudaMalloc: hosts whose own allocator already owns the device's free
// memory, and latency-bound callers that cannot take the device-wide
// synchronisation of cudaMalloc / cudaFree.
//
// The scratch array is a module-level __device__ object of this file's CUDA
// module.  It is reserved on a device when that module is loaded there: at
// the first use of this entry point under CUDA's default lazy module loading,
// at context creation under CUDA_MODULE_LOADING=EAGER; either way it is held
// until the process exits.  Its device address is taken once per device with
// cudaGetSymbolAddress, with that device current.  The work runs on a
// non-blocking stream created once per device, so a call does not
// synchronise with the caller's work on other streams; its host copies are
// from and to the caller's (pageable) buffers, so the call returns only when
// they are done.
#include <cstring>
#include <mutex>
#include <string>

#include "common.cuh"

namespace scatt {
namespace {

constexpr size_t NOALLOC_SCRATCH_BYTES = size_t(64) << 20;   // 64 MiB per device
constexpr int NOALLOC_MAX_ORDER = 1280;
constexpr int NOALLOC_MAX_COUNT = 256;
constexpr int NOALLOC_MAX_DEVICES = 64;
// the size limit stated with the declaration counts 80 bytes per entry
static_assert(sizeof(GjEntry) == 80, "GjEntry layout changed: update the stated scratch formula");

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

std::mutex g_setup_mutex;
void* g_scratch_addr[NOALLOC_MAX_DEVICES] = {};
cudaStream_t g_stream[NOALLOC_MAX_DEVICES] = {};

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

// Byte offsets of the sub-buffers inside the scratch array.
struct Carve {
    size_t A, W, O, P, sig, rid, sigt, st, ent, total;
};

Carve carve(int n, int count) {
    const size_t nn = (size_t)n * n * count;
    Carve c{};
    size_t off = 0;
    auto take = [&](size_t bytes) { const size_t at = off; off += align256(bytes); return at; };
    c.A = take(nn * sizeof(double));
    c.W = take(nn * sizeof(double));
    c.O = take(nn * sizeof(double));
    c.P = take((size_t)2 * n * 64 * count * sizeof(double));
    c.sig = take((size_t)n * count * sizeof(int));
    c.rid = take((size_t)n * count * sizeof(int));
    c.sigt = take((size_t)2 * n * count * sizeof(int));
    c.st = take((size_t)2 * count * sizeof(int));
    c.ent = take((size_t)count * sizeof(GjEntry));
    c.total = off;
    return c;
}

// The per-matrix entry table, written on the device (no host staging).
__global__ void k_noalloc_entries(unsigned char* base, Carve c, int n, int count) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= count) return;
    const size_t nn = (size_t)n * n;
    double* A = reinterpret_cast<double*>(base + c.A);
    double* W = reinterpret_cast<double*>(base + c.W);
    double* O = reinterpret_cast<double*>(base + c.O);
    double* P = reinterpret_cast<double*>(base + c.P);
    int* sig = reinterpret_cast<int*>(base + c.sig);
    int* rid = reinterpret_cast<int*>(base + c.rid);
    int* sigt = reinterpret_cast<int*>(base + c.sigt);
    int* st = reinterpret_cast<int*>(base + c.st);
    GjEntry* ent = reinterpret_cast<GjEntry*>(base + c.ent);
    ent[b] = GjEntry{A + nn * b, W + nn * b, O + nn * b, sig + (size_t)n * b, rid + (size_t)n * b,
                     st + 2 * b, n, n, n, P + (size_t)2 * n * 64 * b, sigt + (size_t)2 * n * b};
}

// Scratch address and stream of the current device; set up once per device.
int scratch_address(unsigned char** out, cudaStream_t* stream) {
    int dev = -1;
    SCATT_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) {
        set_last_error("scatt_inverse_batched_noalloc: device ordinal " + std::to_string(dev) +
                       " outside the supported range");
        return SCATT_ERR_ARG;
    }
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            (void)cudaGetLastError();
            set_last_error(std::string("scatt_inverse_batched_noalloc: cudaGetSymbolAddress: ") +
                           cudaGetErrorString(e));
            return SCATT_ERR_CUDA;
        }
        g_scratch_addr[dev] = p;
    }
    if (!g_stream[dev]) {
        cudaStream_t st = nullptr;
        const cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            (void)cudaGetLastError();
            set_last_error(std::string("scatt_inverse_batched_noalloc: cudaStreamCreate: ") + cudaGetErrorString(e));
            return SCATT_ERR_CUDA;
        }
        g_stream[dev] = st;
    }
    *out = static_cast<unsigned char*>(g_scratch_addr[dev]);
    *stream = g_stream[dev];
    return SCATT_OK;
}

}  // namespace
}  // namespace scatt

using namespace scatt;

extern "C" {

int scatt_inverse_batched_noalloc(int n, int count, const double* A, double* out, int symmetrize,
                                  int* status) {
    if (n <= 0 || count <= 0 || !A || !out) {
        set_last_error("scatt_inverse_batched_noalloc: bad arguments");
        return SCATT_ERR_ARG;
    }
    if (n > NOALLOC_MAX_ORDER || count > NOALLOC_MAX_COUNT) {
        set_last_error("scatt_inverse_batched_noalloc: n " + std::to_string(n) + " / count " +
                       std::to_string(count) + " above the limits " + std::to_string(NOALLOC_MAX_ORDER) +
                       " / " + std::to_string(NOALLOC_MAX_COUNT));
        return SCATT_ERR_SIZE;
    }
    const Carve c = carve(n, count);
    if (c.total > NOALLOC_SCRATCH_BYTES) {
        set_last_error("scatt_inverse_batched_noalloc: needs " + std::to_string(c.total) +
                       " bytes of scratch, the static array holds " + std::to_string(NOALLOC_SCRATCH_BYTES));
        return SCATT_ERR_SIZE;
    }
    SCATT_TRY(require_device());
    unsigned char* base = nullptr;
    cudaStream_t s = nullptr;
    SCATT_TRY(scratch_address(&base, &s));
    const size_t nbytes = (size_t)n * n * count * sizeof(double);
    // the status words (code, first failing column) must start at zero
    SCATT_CUDA_TRY(cudaMemsetAsync(base + c.st, 0, (size_t)2 * count * sizeof(int), s));
    SCATT_CUDA_TRY(cudaMemcpyAsync(base + c.A, A, nbytes, cudaMemcpyHostToDevice, s));
    k_noalloc_entries<<<(count + 127) / 128, 128, 0, s>>>(base, c, n, count);
    SCATT_CUDA_TRY(cudaGetLastError());
    SCATT_COUNT_LAUNCH(1);
    const GjEntry* ent = reinterpret_cast<const GjEntry*>(base + c.ent);
    SCATT_TRY(gj_inverse_selected(ent, count, n, symmetrize != 0, s, false, 64));
    SCATT_CUDA_TRY(cudaMemcpyAsync(out, base + c.O, nbytes, cudaMemcpyDeviceToHost, s));
    int st[2 * NOALLOC_MAX_COUNT];
    SCATT_CUDA_TRY(cudaMemcpyAsync(st, base + c.st, (size_t)2 * count * sizeof(int), cudaMemcpyDeviceToHost, s));
    SCATT_CUDA_TRY(cudaStreamSynchronize(s));
    if (status) std::memcpy(status, st, (size_t)2 * count * sizeof(int));
    for (int b = 0; b < count; ++b) {
        if (st[2 * b] == DEV_SINGULAR) {
            set_last_error("scatt_inverse_batched_noalloc: singular pivot in matrix " + std::to_string(b) +
                           " at column " + std::to_string(st[2 * b + 1]));
            return SCATT_ERR_SINGULAR;
        }
        if (st[2 * b] == DEV_NONFINITE) {
            set_last_error("scatt_inverse_batched_noalloc: non-finite pivot in matrix " + std::to_string(b) +
                           " at column " + std::to_string(st[2 * b + 1]));
            return SCATT_ERR_NONFINITE;
        }
    }
    return SCATT_OK;
}

}  // extern "C"
