/*
 * prr_synth.h -- synthetic ProRes RAW input: frame builder, random tiles,
 * block generator, mosaic generator and encoder.
 *
 * The first group restates the crate's test-support module (feature
 * `testgen`): src/synth.rs (Rng, Spec, frame, random_frame, tile, specs) and
 * the IDCT block generator src/idct.rs:359-459 (testgen::Gen, fnv1a).
 * The second group has no counterpart in the crate, which ships no encoder:
 * a seeded Bayer mosaic generator and an encoder (forward DCT, quantizer,
 * adaptive Golomb-Rice / exp-Golomb entropy coder) that turn a mosaic into a
 * valid frame packet, plus a seeded tile corrupter.
 *
 * Host-only C++ (libprr_synth.so); no CUDA.
 */
#ifndef PRR_SYNTH_H
#define PRR_SYNTH_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* xorshift64* generator, src/synth.rs:9-29. The state is one u64. */
uint64_t prs_rng_new(uint64_t seed);
uint32_t prs_rng_next_u32(uint64_t* state);
uint32_t prs_rng_below(uint64_t* state, uint32_t bound);

/* Spec, src/synth.rs:34-89. has_* flags select the optional fields. */
typedef struct prs_spec {
    uint16_t width, height;
    uint8_t alignment;
    uint8_t pattern; /* header Bayer code */
    uint8_t has_quant_matrix;
    uint8_t has_curve;
    uint8_t quant_matrix[64];
    uint16_t curve[8];
    uint8_t vendor[4];
    uint8_t crop[4];
    uint16_t white_level;
    float wb[2];
    float color_matrix[9];
    float gain;
    uint16_t wb_cct;
    uint8_t valid_tiles;
    uint8_t version; /* written to the header; synth::frame always writes 1 */
} prs_spec;

/* Spec::new(width, height, pattern), src/synth.rs:71-88. */
void prs_spec_new(uint16_t width, uint16_t height, uint8_t pattern, prs_spec* out);
/* specs(rng): the 20 varied specs, src/synth.rs:188-221. Returns the count. */
size_t prs_specs(uint64_t* rng, prs_spec* out, size_t cap);
/* random_frame(spec, rng), src/synth.rs:92-94 and random_tile :158-170.
 * Returns the packet length; writes at most `cap` bytes (call with cap 0
 * to size -- the rng is then NOT advanced). */
size_t prs_random_frame(const prs_spec* spec, uint64_t* rng, uint8_t* out, size_t cap);
/* frame(spec, payload) with one caller payload per tile, concatenated in
 * `tiles` with lengths `tile_lens` (src/synth.rs:99-152). */
size_t prs_frame_from_tiles(const prs_spec* spec, const uint8_t* tiles, const uint32_t* tile_lens,
                            size_t ntiles, uint8_t* out, size_t cap);
/* tile(qscale, streams), src/synth.rs:175-184. */
size_t prs_tile(uint8_t qscale, const uint8_t* const streams[4], const uint32_t lens[4],
                uint8_t* out, size_t cap);

/* Bit writer, the test encoder of src/bits.rs:136-186. ops: kind 0 =
 * symbol(cb=a, value=b); kind 1 = put(value=b, nbits=a). Returns the byte
 * length written (MSB first, zero padded). */
typedef struct prs_bitop {
    uint32_t kind;
    uint32_t a;
    uint32_t b;
} prs_bitop;
size_t prs_bitwrite(const prs_bitop* ops, size_t n, uint8_t* out, size_t cap);

/* testgen::Gen, SplitMix64 block generator (src/idct.rs:363-442): blocks
 * `first`..`first+n` of the stream, continuing from *state. */
uint64_t prs_gen_new(uint64_t seed);
void prs_gen_blocks(uint64_t* state, uint64_t first, size_t n, int16_t* coefs, int16_t* q);
/* FNV-1a over little-endian u16 values (src/idct.rs:445-459). */
uint64_t prs_fnv1a_u16(uint64_t h, const uint16_t* v, size_t n);

/* --- No counterpart in the crate ------------------------------------------ */

/* Seeded Bayer mosaic of linear 12-bit values: three low-frequency 2-D
 * cosines (amplitudes uniform in [amp_lo, amp_hi]) on a 256 offset, scaled
 * per CFA colour by chan_gain (R, G, B), plus Gaussian noise of `sigma`,
 * clipped to [256, white]; a fraction `specular` of sensels is set to white.
 * Rows are generated in parallel with per-row seeds, so the result does not
 * depend on the thread count. */
typedef struct prs_mosaic_params {
    uint32_t width, height;
    uint8_t pattern;
    uint64_t seed;
    float sigma;
    float specular;
    float amp_lo, amp_hi;
    float chan_gain[3];
    uint16_t white;
} prs_mosaic_params;
void prs_mosaic(const prs_mosaic_params* p, uint16_t* out, int threads);

/* Encoder: linear mosaic (width*height, row-major) -> frame packet.
 * The header fields come from `spec` (version, pattern, alignment, matrix,
 * curve, levels, colour). Tile qscale is uniform in [qscale_lo, qscale_hi]
 * drawn from `qscale_seed` per tile (equal bounds: fixed). Returns the
 * packet length, which is larger than `cap` when nothing was written
 * because the buffer is too small, or 0 when a tile would exceed the
 * 65535-byte limit of the size table. */
typedef struct prs_encode_params {
    prs_spec spec;
    uint8_t qscale_lo, qscale_hi;
    uint64_t qscale_seed;
} prs_encode_params;
size_t prs_encode(const prs_encode_params* p, const uint16_t* mosaic, uint8_t* out, size_t cap,
                  int threads);

/* Corrupt about `fraction` of the tiles of a packet in place (seeded):
 * half of them get an invalid tile header (so the decoder skips them), the
 * other half random byte flips inside their streams. The size table is
 * untouched. Writes the chosen tile indices to `tiles` (up to cap) and
 * returns their count. */
size_t prs_corrupt_tiles(uint8_t* packet, size_t len, float fraction, uint64_t seed,
                         uint64_t* tiles, size_t cap);

#ifdef __cplusplus
}
#endif
#endif
