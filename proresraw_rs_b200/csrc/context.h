// context.h -- the library context (device, stream, reusable device and
// pinned host buffers), shared by the single-frame entry points (api.cu) and
// the batch decode (batch.cu).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <string>
#include <vector>

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
    // DNG export: per-tile bit streams, the tiles' look-back words, the
    // packed tiles, their offsets, an error flag, pinned copies of the
    // tiles and offsets, and a linearized image.
    DevBuf<uint32_t> lj_words;
    DevBuf<unsigned long long> lj_lookback;
    DevBuf<uint8_t> lj_out;
    DevBuf<uint64_t> lj_offsets;
    DevBuf<uint32_t> lj_flag;
    HostBuf<uint8_t> lj_hout;
    HostBuf<uint64_t> lj_hoffsets;
    DevBuf<uint16_t> lin;
    uint32_t develop_ctas = 0;  // prr_develop_set_occupancy
    std::map<uint32_t, prr_develop_config> develop_cfgs;  // per frame-size bucket (prr_develop_tune)
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

namespace prr {
// lj92.cu: worst-case stream bytes of one tile, and the tile encoder
// (streams back to back in `out`, offsets[ntiles + 1]; pad_even: each at
// an even offset, a 0 byte after an odd one; *dev_error nonzero when it
// failed).
uint64_t lj92_tile_bound(uint32_t tile);
int lj92_encode(prr_ctx* c, const uint16_t* image, uint32_t width, uint32_t height, uint64_t stride, uint32_t tile,
                uint8_t* out, uint64_t out_cap, uint64_t* dev_offsets, uint32_t* dev_error, bool pad_even);
// dng.cpp: the DNG container -- the bytes before the image data for
// chunks of `sizes` bytes (each then padded to an even length), the whole
// file around chunks in host memory, and file objects.
int dng_prefix(const prr_header* header, const prr_dng_clip* clip, int samples, int compression,
               const std::vector<uint32_t>& sizes, std::vector<uint8_t>& prefix);
int dng_assemble(const prr_header* header, const prr_dng_clip* clip, int samples, int compression,
                 const uint8_t* data, const uint64_t* offsets, size_t nchunks, prr_dng_file** out);
prr_dng_file* dng_file_new(size_t bytes);
uint8_t* dng_file_bytes(prr_dng_file* f);
}  // namespace prr
