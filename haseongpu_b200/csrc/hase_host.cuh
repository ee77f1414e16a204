// hase_host.cuh -- host-side helpers shared by the translation units of
// libhase_b200.so: the thread-local error message behind
// hase_last_error_message(), CUDA error mapping, and an owning device buffer.
#pragma once

#include "hase_b200.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>

namespace hase {

// Records the message returned by hase_last_error_message() and returns st.
hase_status fail(hase_status st, const char* fmt, ...);

template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    cudaError_t ensure(size_t count) {
        if (count <= n) return cudaSuccess;
        release();
        cudaError_t e = cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T));
        if (e == cudaSuccess) n = count;
        else p = nullptr;
        return e;
    }
};

}  // namespace hase

#define HASE_CUDA(call)                                                                                  \
    do {                                                                                                 \
        cudaError_t e_ = (call);                                                                         \
        if (e_ != cudaSuccess) {                                                                         \
            return ::hase::fail(e_ == cudaErrorMemoryAllocation ? HASE_OUT_OF_MEMORY : HASE_CUDA_ERROR,    \
                                "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__);    \
        }                                                                                                \
    } while (0)

#define HASE_TRY(expr)               \
    do {                             \
        hase_status s_ = (expr);     \
        if (s_ != HASE_OK) return s_; \
    } while (0)
