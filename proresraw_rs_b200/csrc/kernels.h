// kernels.h -- host-side launchers of the library's CUDA kernels.
#pragma once

#include <cuda.h>
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
// Batch decode: the frames of a batch in one persistent launch that drains
// a queue of work items: first the entropy chunks of every frame (a chunk is
// the streams of threads / 4 consecutive tiles), then the transform
// segments of every frame (tile row x 256-sensel segment). A segment waits
// for the chunk flags of its tiles, set to the batch's epoch.
struct BatchFrame {
    FrameDesc d;            // counts / pairs point into the batch scratch
    uint32_t* tile_off;     // ntiles + 1 offsets
    prr_dev_status* st;
    uint32_t* skipped;      // ntiles entries
    uint16_t* out;
    uint32_t shift;         // 0: full resolution; 1..3: reduced by 2^shift
    uint32_t idct;          // full resolution
    uint32_t greens;        // reduced
    uint32_t lc;            // log2 coefficients decoded per block
    uint32_t ent_begin;     // first entropy item (chunk) of the frame
    uint32_t seg_begin;     // first transform item of the frame, counted after all chunks
    uint32_t pad[2];
};

struct BatchQueue {
    uint32_t head;   // next work item
    uint32_t epoch;  // batch sequence number; chunk flags hold it when done
    uint32_t error;  // a wait for a chunk ran out of time
    uint32_t pad;
};

// Sizes of the current batch, uploaded with its frames, so that one launch
// (or one captured graph) serves every batch that fits the buffers.
struct BatchHeader {
    uint32_t nframes;
    uint32_t ent_items;      // chunks of all frames
    uint32_t seg_items;      // segments of all frames
    uint32_t wait_limit_us;  // a segment's wait for a chunk flag (0: kChunkWaitNs)
    uint32_t drop_item;      // a chunk claimed but never decoded nor flagged (tests), or NO_TILE
    uint32_t streams_per_thread;  // of an entropy item: 1, 2 or 4 (tiles per item: 64 x it)
    uint32_t pad[2];
};

struct BatchDesc {
    const BatchHeader* hdr;
    const BatchFrame* frames;
    BatchQueue* q;
    uint32_t* flags;  // one per chunk
    uint32_t stage_bytes;
};

constexpr uint32_t kBatchThreads = 256;
// Tiles of an entropy item: streams_per_thread x kBatchThreads streams,
// four a tile.
constexpr uint32_t kBatchMaxStreamsPerThread = 4;
__host__ __device__ constexpr uint32_t batch_tiles_per_item(uint32_t streams_per_thread) {
    return streams_per_thread * kBatchThreads / 4;
}
constexpr uint32_t kBatchMaxStageBytes = 96 * 1024;
// Dynamic shared memory of the batch kernel for a packet stage of
// stage_bytes (<= kBatchMaxStageBytes), and the CTAs per SM that fit.
size_t batch_smem_bytes(uint32_t stage_bytes);
cudaError_t batch_prepare_device();
cudaError_t batch_max_ctas_per_sm(uint32_t stage_bytes, int* ctas);
cudaError_t launch_batch_tile_index(const BatchDesc& b, uint32_t grid, cudaStream_t s);
cudaError_t launch_batch_decode(const BatchDesc& b, uint32_t ctas, cudaStream_t s);

cudaError_t launch_transform_blocks(int kind, const int16_t* coefs, const int16_t* q,
                                    uint16_t* out, size_t n, cudaStream_t s);
cudaError_t launch_decode_components(const uint8_t* packet, const uint32_t* off,
                                     const uint32_t* len, size_t n, int log2_blocks,
                                     int log2_coefs, int16_t* coefs, cudaStream_t s);
cudaError_t launch_decode_components_events(const uint8_t* packet, const uint32_t* off,
                                            const uint32_t* len, size_t n, int log2_blocks, int log2_coefs,
                                            int staged, uint32_t* lists, int16_t* coefs, uint32_t* flags,
                                            cudaStream_t s);

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
    // Non-null: develop only the 32x32 tiles whose byte is nonzero (row-major
    // over the tile grid).
    const unsigned* tile_mask;
    // Nonzero: at most this many CTAs per SM (shared memory reserved per
    // CTA), leaving room for kernels of other streams.
    uint32_t ctas_per_sm;
    // Set by launch_develop: interior tiles load their code values by TMA.
    uint32_t use_tma;
    // Output tile shape (0, 0: 32 x 32); see develop_shape_supported.
    uint32_t tile_w, tile_h;
};

constexpr int kDevelopTile = 32;
// Devices a process may use with the library's per-device launch caches.
constexpr int kMaxDevices = 64;

// Argument checks and kernel descriptor of develop_into / develop_planar_into
// (api.cu), and output_matrix (src/demosaic.rs:138-153).
int build_develop_desc(const prr_header* h, const prr_params* params, int stage, const uint16_t* dev_samples,
                       int layout, float* r, float* g, float* b, size_t out_len, DevelopDesc* out);
void output_matrix(const prr_header* h, int exposure, float* m);

cudaError_t launch_linearize(const uint16_t* codes, uint32_t stride, int w, int h,
                             const uint32_t* c0, const uint32_t* delta, uint16_t* out,
                             cudaStream_t s);
cudaError_t launch_develop(const DevelopDesc& d, cudaStream_t s);
// The develop tile shapes launch_develop instantiates: 32x32 (default),
// 32x16 and 64x16.
bool develop_shape_supported(uint32_t tile_w, uint32_t tile_h);
// Whether the develop's parameters keep every quotient of its green and
// chroma passes in the range of the paired division (fastdiv.cuh).
bool develop_fast_division_ok(const DevelopDesc& d);
cudaError_t launch_div_rn_pairs(const float* a, const float* b, float* q, size_t n, cudaStream_t s);
cudaError_t launch_sqrt_rn_check(int e_min, int e_max, unsigned long long* mismatches, cudaStream_t s);
cudaError_t launch_div_rn_check(uint32_t b_first, uint32_t b_count, unsigned long long* mismatches,
                                cudaStream_t s);
// learned.cu: a 2-D tensor map of 16-bit elements (cuTensorMapEncodeTiled
// through the runtime's driver entry point).
cudaError_t encode_u16_map_2d(CUtensorMap* map, const void* base, uint64_t width, uint64_t height,
                              uint64_t row_bytes, uint32_t box_w, uint32_t box_h);

}  // namespace prr
