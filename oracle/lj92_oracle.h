/*
 * lj92_oracle.h -- CPU restatement of the DNG export's lossless JPEG tile
 * encoding (examples/prr2dng/lj92.rs and the tile cut of
 * examples/prr2dng/dng.rs:115-127).
 *
 * TEST INFRASTRUCTURE ONLY (built into libprr_oracle.so): the checker of
 * the library's device LJ92 encoder, and the timed CPU baseline of the DNG
 * workload. Never linked into the product.
 *
 * Parity: the reference is Rust and cannot be built in this image, so no
 * reference-generated streams exist. The restatement is pinned by the
 * reference's own tests of this encoder (lj92.rs:249-399: round trips of
 * random and extreme samples through a decoder, a flat tile's size bound,
 * the Huffman table of a skewed histogram) run against it, and by a
 * decoder in the tests that reads its streams back to the samples.
 */
#ifndef LJ92_ORACLE_H
#define LJ92_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* lj92::encode (lj92.rs:14-69): the lossless JPEG stream of `samples`,
 * width x height row-major, `components` interleaved components. Returns 0,
 * or -1 when `cap` is too small (*len then holds the size needed) or the
 * arguments are invalid. */
int orc_lj92_encode(const uint16_t* samples, size_t width, size_t height, size_t components, uint8_t* out,
                    size_t cap, size_t* len);

/* HuffmanTable::optimal (lj92.rs:96-202) of a histogram over categories
 * 0..16: BITS (counts[16]), HUFFVAL (values, *nvalues of them) and each
 * category's code and length (length 0: unused). */
void orc_lj92_huffman(const uint64_t histogram[17], uint8_t counts[16], uint8_t values[17], int* nvalues,
                      uint16_t codes[17], uint8_t lengths[17]);

/* dng::tile (dng.rs:115-127): the tile x tile square at (left, top) of a
 * width x height image whose rows are `stride` samples apart; sensels past
 * the right or bottom edge repeat the nearest edge sensel of the same CFA
 * colour. width and height must be at least 2. */
int orc_dng_tile(const uint16_t* values, size_t width, size_t height, size_t stride, size_t left, size_t top,
                 size_t tile, uint16_t* out);

/* Every tile of the image, row by row, encoded as dng::write does
 * (dng.rs:95-103: lj92::encode(tile, T, T, 2) per tile, tiles in parallel
 * on `threads` threads, 0 = all cores). Tile i's stream is written at
 * out + offsets[i]; offsets has ntiles + 1 entries (the last = total
 * bytes). Returns 0, or -1 when `cap` is too small. */
int orc_lj92_tiles(const uint16_t* values, size_t width, size_t height, size_t stride, size_t tile, int threads,
                   uint8_t* out, size_t cap, uint64_t* offsets);

#ifdef __cplusplus
}
#endif
#endif
