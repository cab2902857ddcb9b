// context.h -- the library context (device, stream, reusable device and
// pinned host buffers), shared by the single-frame entry points (api.cu) and
// the batch decode (batch.cu).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "../../include/prr.h"

template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t cap = 0;  // elements
    cudaError_t ensure(size_t n) {
        if (n <= cap) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        cudaError_t e = cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T));
        if (e == cudaSuccess) cap = n;
        return e;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
};

template <class T>
struct HostBuf {
    T* p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t n) {
        if (n <= cap) return cudaSuccess;
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
        cudaError_t e = cudaMallocHost(&p, std::max<size_t>(n, 1) * sizeof(T));
        if (e == cudaSuccess) cap = n;
        return e;
    }
    void release() {
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
    }
};

namespace prr {
struct BatchState;  // batch.cu
void batch_state_destroy(BatchState* b);
struct LearnedState;  // learned.cu
void learned_state_destroy(LearnedState* s);
}  // namespace prr

struct prr_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    DevBuf<uint8_t> pkt;
    HostBuf<uint8_t> hpkt;
    DevBuf<uint8_t> scratch;  // decode scratch (tile offsets, stream counts, coefficient lists)
    DevBuf<uint32_t> skipped;
    DevBuf<prr_dev_status> status;
    HostBuf<prr_dev_status> hstatus;
    HostBuf<uint32_t> hskipped;
    DevBuf<uint16_t> samples;
    DevBuf<float> planes;
    prr::BatchState* batch = nullptr;
    prr::LearnedState* learned = nullptr;
    std::string last_error;

    int cuda(cudaError_t e) {
        if (e == cudaSuccess) return PRR_OK;
        last_error = cudaGetErrorString(e);
        return PRR_ERR_CUDA;
    }
    int use_device() { return cuda(cudaSetDevice(device)); }
};

#define PRR_TRY(expr)                     \
    do {                                  \
        int _rc = (expr);                 \
        if (_rc != PRR_OK) return _rc;    \
    } while (0)
