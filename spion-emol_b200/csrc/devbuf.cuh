// devbuf.cuh -- RAII device buffer used by the host orchestration.
#pragma once

#include <vector>

#include "common.cuh"

namespace scatt {

template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
    DevBuf& operator=(DevBuf&& o) noexcept {
        if (this != &o) { release(); p = o.p; n = o.n; o.p = nullptr; o.n = 0; }
        return *this;
    }
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    int alloc(size_t count) {
        release();
        if (count == 0) count = 1;
        cudaError_t e = cudaMalloc(&p, count * sizeof(T));
        if (e != cudaSuccess) {
            (void)cudaGetLastError();
            p = nullptr;
            set_last_error(std::string("device allocation of ") +
                           std::to_string(count * sizeof(T)) + " bytes failed: " +
                           cudaGetErrorString(e));
            return SCATT_ERR_OOM;
        }
        n = count;
        return SCATT_OK;
    }
    int zero(cudaStream_t s = 0) {
        SCATT_CUDA_TRY(cudaMemsetAsync(p, 0, n * sizeof(T), s));
        return SCATT_OK;
    }
    int upload(const std::vector<T>& h, cudaStream_t s = 0) {
        if (n < h.size()) SCATT_TRY(alloc(h.size()));
        if (!h.empty())
            SCATT_CUDA_TRY(cudaMemcpyAsync(p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, s));
        return SCATT_OK;
    }
    int upload(const T* h, size_t count, cudaStream_t s = 0) {
        if (n < count) SCATT_TRY(alloc(count));
        if (count)
            SCATT_CUDA_TRY(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
        return SCATT_OK;
    }
};

}  // namespace scatt
