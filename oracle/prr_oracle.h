/*
 * prr_oracle.h -- C ABI of the CPU oracle.
 *
 * TEST INFRASTRUCTURE ONLY. This library is a plain C++ restatement of the
 * CPU decode / linearize / develop path of the proresraw_rs crate
 * (src/bits.rs, codebook.rs, coefficients.rs, idct.rs, header.rs, tile.rs,
 * decoder.rs, reduced.rs, curve.rs, demosaic.rs). It exists to check the
 * CUDA product path and to serve as the timed CPU baseline. Only the tests,
 * the smoke check and the CPU-baseline leg of bench.py may load it; the
 * product library never links or calls it.
 *
 * Status codes follow the crate's `Error` enum (src/error.rs:6-63) with the
 * same numbering as include/prr.h.
 */
#ifndef PRR_ORACLE_H
#define PRR_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    ORC_OK = 0,
    ORC_ERR_TRUNCATED = -1,
    ORC_ERR_FRAME_SIZE_MISMATCH = -2,
    ORC_ERR_BAD_QUANT_MATRIX = -3,
    ORC_ERR_BAD_CURVE = -4,
    ORC_ERR_UNEXPECTED_CURVE = -5,
    ORC_ERR_BAD_TAG = -6,
    ORC_ERR_HEADER_TOO_SHORT = -7,
    ORC_ERR_UNSUPPORTED_VERSION = -8,
    ORC_ERR_BAD_DIMENSIONS = -9,
    ORC_ERR_BAD_ALIGNMENT = -10,
    ORC_ERR_TILE_OUT_OF_BOUNDS = -11,
    ORC_ERR_BAD_TILE_HEADER = -12,
    ORC_ERR_BUFFER = -20,
};

/* Payload of an error, the fields of the matching `Error` variant. */
typedef struct orc_error {
    int32_t code;
    char what[32];       /* Truncated::what */
    uint64_t needed;     /* Truncated::needed */
    uint64_t available;  /* Truncated::available */
    uint32_t declared;   /* FrameSizeMismatch::declared */
    uint64_t actual;     /* FrameSizeMismatch::actual */
    uint64_t index;      /* BadQuantMatrix::index, TileOutOfBounds/BadTileHeader::tile */
    uint32_t value;      /* BadQuantMatrix::value, UnsupportedVersion, BadAlignment, HeaderTooShort */
    uint16_t width, height;
    uint16_t curve[8];
    uint8_t tag[4];
} orc_error;

/* FrameHeader (src/header.rs:112-146). */
typedef struct orc_header {
    uint8_t version;
    uint8_t vendor[4];
    uint8_t bayer_pattern; /* header code 0 RGGB, 1 GRBG, 2 GBRG, 3 BGGR */
    uint16_t width, height;
    uint8_t crop[4]; /* left, right, top, bottom */
    uint16_t white_level;
    uint16_t wb_cct;
    uint16_t flags;
    uint8_t alignment;
    uint8_t pad0;
    float wb_red, wb_blue;
    float color_matrix[9];
    float gain;
    uint8_t quant_matrix[64];
    uint16_t curve[8];
} orc_header;

/* DemosaicParams (src/demosaic.rs:57-74). */
typedef struct orc_params {
    int32_t cfa_phase;
    int32_t black;
    float one_over_range;
    float noise[3];
    float clip[2];
    float black_over_range;
    float wb[2];
} orc_params;

/* --- bits.rs / codebook.rs / coefficients.rs --------------------------------- */
void orc_codeword(uint32_t p, uint16_t cb, uint32_t* value, uint32_t* len);
/* Read up to `n` symbols with the given codebooks from a stream; returns the
 * number read before the view went to zero. */
int orc_read_symbols(const uint8_t* data, size_t len, size_t align, const uint16_t* cbs,
                     size_t n, uint32_t* out);
void orc_decode_component_reduced(const uint8_t* data, size_t len, size_t align,
                                  uint8_t log2_blocks, uint8_t log2_coefs, int16_t* coefs);

/* --- idct.rs ----------------------------------------------------------------- */
int16_t orc_dequantize(int16_t coef, int16_t q);
void orc_apple_block(const int16_t* coefs, const int16_t* q, uint16_t* out);
void orc_ffmpeg_block(const int16_t* coefs, const int16_t* q, uint16_t* out);
void orc_apple_block_4x4(const int16_t* coefs, const int16_t* q, uint16_t* out);
void orc_apple_block_2x2(const int16_t* coefs, const int16_t* q, uint16_t* out);
uint16_t orc_output_code(float v);
uint16_t orc_code_value(int32_t centered);
/* Apple or FFmpeg transform of n blocks (idct: 0 Apple, 1 FFmpeg). */
void orc_transform_blocks(int idct, const int16_t* coefs, const int16_t* q, uint16_t* out,
                          size_t n);

/* --- curve.rs ---------------------------------------------------------------- */
uint16_t orc_curve_linearize(const uint16_t* curve, uint16_t code);

/* --- header.rs / decoder.rs / tile.rs --------------------------------------- */
int orc_header_len(const uint8_t* pkt, size_t len, size_t* out, orc_error* err);
int orc_parse_header(const uint8_t* pkt, size_t len, orc_header* out, orc_error* err);
/* parse_frame: header, grid and tile slices. `tile_off`/`tile_len` may be
 * NULL; otherwise they hold `*ntiles` entries (call once with NULL to size). */
int orc_parse_frame(const uint8_t* pkt, size_t len, orc_header* hdr, size_t* ntiles,
                    size_t* tiles_per_row, size_t* tile_rows, uint64_t* tile_off,
                    uint64_t* tile_len, uint8_t* max_qscale, orc_error* err);
int orc_tile_parse(const uint8_t* data, size_t len, size_t index, uint8_t* qscale,
                   uint64_t* stream_off, uint64_t* stream_len);
/* Geometry of the tiles of one grid row: x in sensels and log2 blocks. */
size_t orc_grid_row(size_t width, size_t height, uint8_t alignment, size_t* x,
                    uint8_t* log2_blocks);

/* decode_frame_with: samples hold coded_w*coded_h values; skipped holds up to
 * `skipped_cap` indices. threads 0 = all cores. */
int orc_decode_frame(const uint8_t* pkt, size_t len, int idct, uint16_t* samples,
                     size_t samples_len, uint64_t* skipped, size_t skipped_cap,
                     size_t* n_skipped, uint8_t* max_qscale, orc_header* hdr, int threads,
                     orc_error* err);
/* decode_frame_reduced_with: scale 1 half, 2 quarter, 3 eighth (log2 factor);
 * greens 0 first, 1 average. */
int orc_decode_frame_reduced(const uint8_t* pkt, size_t len, int log2_factor, int greens,
                             uint16_t* samples, size_t samples_len, uint64_t* skipped,
                             size_t skipped_cap, size_t* n_skipped, uint8_t* max_qscale,
                             orc_header* hdr, int threads, orc_error* err);
/* Frame::linearize_into: visible width*height values from coded samples. */
int orc_linearize(const orc_header* hdr, const uint16_t* samples, uint16_t* out,
                  size_t out_len, int threads);

/* --- demosaic.rs ------------------------------------------------------------- */
void orc_params_with_white_balance(const orc_header* hdr, uint32_t quantizer, float red,
                                   float blue, orc_params* out);
void orc_output_matrix(const orc_header* hdr, int exposure, float* m9);
/* develop_into (interleaved) or develop_planar_into: stage 0 Demosaiced,
 * 1 WhiteBalanced, 2 Rec2020. `planar` selects the output form; for
 * interleaved only `r` is used (3*w*h floats). */
int orc_develop(const orc_header* hdr, const uint16_t* samples, const orc_params* p,
                int stage, int planar, float* r, float* g, float* b, size_t out_len,
                int threads);
/* The public passes: green_pass on linear values, chroma_pass, apply_matrix. */
void orc_green_pass(const uint16_t* linear, size_t w, size_t h, const orc_params* p,
                    float* out2);
void orc_chroma_pass(const float* green2, size_t w, size_t h, const orc_params* p,
                     float* out3);
void orc_apply_matrix(const float* rgb, size_t n_px, const float* m9, float* out);

#ifdef __cplusplus
}
#endif
#endif
