// kernels.h -- host-side launchers of the library's CUDA kernels.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "../../include/prr.h"

namespace prr {

constexpr uint32_t NO_TILE = 0xFFFFFFFFu;

// Per-frame constants of the decode kernels.
struct FrameDesc {
    const uint32_t* words;  // the packet, 4-byte aligned
    uint32_t len;           // packet bytes
    uint32_t table_off;     // byte offset of the tile size table
    uint32_t ntiles, tiles_per_row, tile_rows;
    uint32_t columns;       // 16-sensel columns (coded_width / 16)
    uint32_t alignment;
    uint32_t coded_w;
    uint32_t segs_per_row;  // 256-sensel segments per tile row
    uint32_t phase[4];      // phase of stream s: 2 * row parity + column parity
    uint32_t curve_c0[8];   // linearization segments (reduced decode)
    uint32_t curve_delta[8];
    uint8_t qmat[64];
    // Split decode (k_entropy, then the transform kernel): per-stream entry
    // counts and (position, value) lists. Both null: the fused kernels
    // entropy-decode inside the transform CTA.
    uint32_t* counts;
    uint32_t* pairs;
};

// Scratch of the split decode for a frame: tile offsets, then per-stream
// counts, then the coefficient lists, each 256-byte aligned.
struct DecodeScratch {
    size_t tile_off, counts, pairs, total;
};
DecodeScratch decode_scratch_layout(uint32_t ntiles, uint32_t coded_w, uint32_t coded_h);

FrameDesc make_frame_desc(const prr_frame_info& info, const uint8_t* dev_packet);

// Dense linear launches (grid sizing, counters) share this.
void count_launch(uint32_t n = 1);

cudaError_t launch_tile_index(const FrameDesc& d, uint32_t* tile_off, prr_dev_status* st,
                              cudaStream_t s);
cudaError_t launch_decode_full(const FrameDesc& d, int idct, const uint32_t* tile_off,
                               prr_dev_status* st, uint32_t* skipped, uint16_t* out,
                               cudaStream_t s);
cudaError_t launch_decode_reduced(const FrameDesc& d, int shift, int greens,
                                  const uint32_t* tile_off, prr_dev_status* st, uint32_t* skipped,
                                  uint16_t* out, cudaStream_t s);
cudaError_t launch_transform_blocks(int kind, const int16_t* coefs, const int16_t* q,
                                    uint16_t* out, size_t n, cudaStream_t s);
cudaError_t launch_decode_components(const uint8_t* packet, const uint32_t* off,
                                     const uint32_t* len, size_t n, int log2_blocks,
                                     int log2_coefs, int16_t* coefs, cudaStream_t s);

// Develop / linearize.
struct DevelopDesc {
    const uint16_t* codes;
    uint32_t stride;  // coded width
    int32_t w, h;
    uint32_t curve_c0[8], curve_delta[8];
    int32_t cfa;
    int32_t black;
    float one_over_range;
    float green_off;   // black as f32 * one_over_range (green pass)
    float chroma_off;  // black_over_range (chroma pass)
    float noise[3];
    float clip[2];
    float wb[2];
    int32_t has_matrix;
    float m[9];
    int32_t layout;  // PRR_INTERLEAVED / PRR_PLANAR
    float* r;
    float* g;
    float* b;
};

cudaError_t launch_linearize(const uint16_t* codes, uint32_t stride, int w, int h,
                             const uint32_t* c0, const uint32_t* delta, uint16_t* out,
                             cudaStream_t s);
cudaError_t launch_develop(const DevelopDesc& d, cudaStream_t s);

}  // namespace prr
