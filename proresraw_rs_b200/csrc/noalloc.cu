// noalloc.cu -- a frame decode that allocates nothing.
//
// Some callers cannot allocate device memory at the moment they decode a
// frame: plug-ins whose host application owns all device memory and hands
// them only the input and output buffers, and real-time ingest or playback
// loops where a cudaMalloc/cudaFree would synchronize the device and stall
// the other work on it, or could fail outright because another allocator
// has already reserved the memory. prr_decode_noalloc serves them: the only
// scratch the decode needs beyond its inputs and outputs, the table of tile
// byte offsets, lives in a fixed array compiled into the library.

#include <cuda_runtime.h>

#include <mutex>

#include "../../include/prr.h"
#include "kernels.h"

namespace {

// Scratch of the tile-offset table: one u32 per tile plus the end offset.
// It exists once per device that loads the library and stays allocated
// until the process exits. Every call shares it.
constexpr uint32_t kMaxTiles = PRR_NOALLOC_MAX_TILES;
static __device__ __align__(256) uint32_t g_tile_off[kMaxTiles + 1];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
void* g_scratch[kMaxDevices] = {};

// The device address of g_tile_off on `device`, looked up once per device
// with that device current. Host code cannot pass &g_tile_off to a kernel:
// on the host the name stands for a host-side shadow, not device memory.
// The cached address belongs to the device's primary context; it is not
// valid after cudaDeviceReset (the library does not support that).
int scratch_for(int device, uint32_t** out) {
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_scratch[device]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_tile_off) != cudaSuccess || p == nullptr) {
            cudaGetLastError();
            return PRR_ERR_CUDA;
        }
        g_scratch[device] = p;
    }
    *out = static_cast<uint32_t*>(g_scratch[device]);
    return PRR_OK;
}

// The decode proper, with `device` current.
int decode_on_device(int device, cudaStream_t s, const prr_frame_info* info, const uint8_t* dev_packet,
                     int idct, uint16_t* dev_samples, prr_dev_status* dev_status, uint32_t* dev_skipped) {
    uint32_t* tile_off = nullptr;
    const int rc = scratch_for(device, &tile_off);
    if (rc != PRR_OK) return rc;
    const prr::FrameDesc d = prr::make_frame_desc(*info, dev_packet);
    if (prr::launch_tile_index(d, tile_off, dev_status, s) != cudaSuccess) return PRR_ERR_CUDA;
    if (prr::launch_decode_full(d, idct, tile_off, dev_status, dev_skipped, dev_samples, s) != cudaSuccess)
        return PRR_ERR_CUDA;
    return PRR_OK;
}

}  // namespace

extern "C" int prr_decode_noalloc(int device, void* cuda_stream, const prr_frame_info* info,
                                  const uint8_t* dev_packet, int idct, uint16_t* dev_samples,
                                  prr_dev_status* dev_status, uint32_t* dev_skipped) {
    // Argument checks come before any CUDA call.
    if (device < 0 || device >= kMaxDevices) return PRR_ERR_INVALID;
    if (!info || !dev_packet || !dev_samples || !dev_status || !dev_skipped) return PRR_ERR_INVALID;
    if ((reinterpret_cast<uintptr_t>(dev_packet) & 3) != 0) return PRR_ERR_INVALID;
    if (idct != PRR_IDCT_APPLE && idct != PRR_IDCT_FFMPEG) return PRR_ERR_INVALID;
    if (info->ntiles > kMaxTiles) return PRR_ERR_SCRATCH_LIMIT;
    // The caller's current device is put back before returning: a plug-in
    // host that owns the device context keeps its own current device.
    int caller = -1;
    if (cudaGetDevice(&caller) != cudaSuccess) {
        cudaGetLastError();
        return PRR_ERR_CUDA;
    }
    if (caller != device && cudaSetDevice(device) != cudaSuccess) {
        cudaGetLastError();
        return PRR_ERR_CUDA;
    }
    const int rc = decode_on_device(device, static_cast<cudaStream_t>(cuda_stream), info, dev_packet, idct,
                                    dev_samples, dev_status, dev_skipped);
    if (caller != device && cudaSetDevice(caller) != cudaSuccess) {
        cudaGetLastError();
        return rc != PRR_OK ? rc : PRR_ERR_CUDA;
    }
    return rc;
}
