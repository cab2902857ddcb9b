/*
 * sg_oracle.h -- CPU reference of the learned demosaic surrogate.
 *
 * TEST INFRASTRUCTURE ONLY (built into libprr_oracle.so beside the crate
 * restatement): the checker of the library's surrogate kernels. The crate
 * has no surrogate; this file states the network the library implements,
 * in plain loops:
 *
 *  input   a half-resolution image of 16 channels, one pixel per 2x2 Bayer
 *          quad. From the quad's red, green on the red row, green on the
 *          blue row and blue (normalized linear values as the plain develop
 *          computes them, red and blue times their white-balance gains) and
 *          its mean green gm: 4 (red - gm), 4 (green r - gm), 4 (green b - gm),
 *          4 (blue - gm), a noise channel 64 * sqrt(variance(gm)) from the
 *          plain develop's noise model, gm, 4 gx, 4 gy and 4 lap, where gx,
 *          gy are half the differences of the neighbouring quads' gm (east -
 *          west, south - north; the grid clamped at its edges) and lap is gm
 *          minus the mean of those four; then 7 zero channels. Small values
 *          in bf16 keep the fine detail the output needs;
 *  layers  conv 3x3 16->32, five conv 3x3 32->32, each + bias and ReLU,
 *          stored as bf16; head conv 3x3 32->16 (12 used) + bias, f32.
 *          Zero padding outside the image at every layer; products of bf16
 *          values accumulated in f32;
 *  frame   the network works on the picture mirrored horizontally when red
 *          sits in the right column of a quad and vertically when it sits in
 *          the bottom row, so every Bayer pattern reaches it as RGGB;
 *  output  full-resolution RGB: head channel c*4 + 2*sy + sx of network quad
 *          (i, j) plus the quad's own colour (red, mean green, blue) gives
 *          network pixel (2i + sx, 2j + sy), mirrored back to the picture;
 *          min(., 1) and the Rec.2020 matrix for that stage, as the plain
 *          develop applies them. The loss and its gradient are stated in the
 *          network frame (targets mirrored into it).
 *
 * Parameters are f32, layer by layer: weights [cout][cin][9] (tap = 3*dy +
 * dx), then bias [cout].
 */
#ifndef SG_ORACLE_H
#define SG_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#include "prr_oracle.h"

#ifdef __cplusplus
extern "C" {
#endif

size_t orc_sg_param_count(void);

/* Pack a decoded frame (code values, coded stride) into the surrogate input
 * [16][hq][wq] (bf16-rounded) and the quad colours base [3][hq][wq]. */
int orc_sg_pack(const orc_header* hdr, const uint16_t* samples, const orc_params* params, float* in16,
                float* base3);

/* Forward over one image of h x w pixels. acts (nullable) receives the six
 * hidden activations [6][32][h][w]; head receives [16][h][w]. round_bf16 = 0
 * keeps every value in f32 (for finite-difference checks). */
void orc_sg_forward(const float* in16, int h, int w, const float* params, int round_bf16, float* acts,
                    float* head);

/* Full-resolution RGB from head and base (planar, width x height visible
 * pixels, mirrored back from the network frame of Bayer phase `cfa`); m9
 * NULL for the white-balanced stage. */
void orc_sg_output(const float* head, const float* base3, int hq, int wq, int width, int height, int cfa,
                   const float* m9, float* r, float* g, float* b);

/* Mean squared error of the unclipped output against target planes over the
 * visible pixels, and its gradient with respect to the head. */
double orc_sg_loss(const float* head, const float* base3, int hq, int wq, int width, int height,
                   const float* tr, const float* tg, const float* tb, float* dhead);

/* Gradient of the loss with respect to the parameters, from the forward's
 * activations and the head gradient. */
void orc_sg_backward(const float* in16, int h, int w, const float* params, const float* acts,
                     const float* dhead, float* dparams);

#ifdef __cplusplus
}
#endif

#endif
