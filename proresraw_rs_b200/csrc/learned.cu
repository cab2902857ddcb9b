// learned.cu -- the learned demosaic surrogate: a small convolutional network
// that develops a decoded frame to white-balanced (or Rec.2020) RGB, run on
// the 5th-generation tensor cores, with its training on the device. No
// counterpart in the crate: the plain develop (develop.cu) is its reference,
// its training target and its per-tile fallback.
//
// Network (the CPU restatement in the oracle states the same):
//  input   half resolution, one pixel per 2x2 Bayer quad, 16 channels. From
//          the quad's red, two greens and blue (normalized linear values as
//          the plain develop computes them, red and blue times their
//          white-balance gains) and its mean green gm: 4 (each colour - gm),
//          a noise channel 64 * sqrt of the plain develop's noise variance at
//          gm, gm, 4 gx, 4 gy, 4 lap (half differences of the neighbouring
//          quads' gm, east - west and south - north, and gm minus their mean;
//          the quad grid clamped at its edges), 7 zero channels. The small
//          differences keep in bf16 the detail the output needs;
//  layers  conv 3x3 16->32, five conv 3x3 32->32 (bias, ReLU, bf16), head
//          conv 3x3 32->16 (12 used; bias, f32); zero padding at every layer;
//          bf16 products accumulated in f32 (tcgen05.mma kind::f16);
//  frame   the network sees the picture mirrored horizontally when red sits
//          in the right column of a quad and vertically when it sits in the
//          bottom row: every Bayer pattern reaches it as RGGB;
//  output  head channel c*4 + 2*sy + sx of a network-frame quad plus the
//          quad's colour (red, mean green, blue) is network pixel
//          (2i + sx, 2j + sy), mirrored back to the picture; min(., 1), then
//          the Rec.2020 matrix for that stage.
//
// Data layouts: activations bf16 in channel chunks, [image][C/8][H][W][8]
// (16 bytes per pixel and chunk: a run of 8 pixels of one chunk is one
// 8 x 16-byte core matrix of the tensor core's K-major operand layout);
// head, gradients and colours f32 planar [image][C][H][W].
//
// Convolution on the tensor cores (k_sg_rows): a CTA streams the input rows
// of a 128-pixel strip through shared memory; for each row, column offset
// and 16-channel half, one thread issues tcgen05.mma.cta_group::1.kind::f16
// with M = 128 (the strip's pixels: A is the row, its start address moved by
// the column offset), K = 16 and N = 3 x cout: B stacks the three kernel
// rows' weights, so one MMA adds the row's products to the three output rows
// it touches, whose accumulators are consecutive slots of a ring in tensor
// memory (the first MMA into a slot overwrites it). A finished output row
// is read back with tcgen05.ld (a warp per 32 lanes), biased, rectified and
// stored as bf16 chunks (or the f32 head, or the develop output).
//
// Backward (training only) runs on the CUDA cores in f32: the gradient of
// each layer's input through the ReLU, and weight and bias gradients reduced
// per CTA and added with atomics. Adam keeps f32 master weights; the tensor
// core copy is re-packed to bf16 before each forward.

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <climits>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/prr.h"
#include "context.h"
#include "device_common.cuh"
#include "kernels.h"

namespace prr {
namespace sg {

constexpr int kIn = 16, kHid = 32, kHead = 16, kLayers = 7;
__host__ __device__ constexpr int cin_of(int l) { return l == 0 ? kIn : kHid; }
__host__ __device__ constexpr int cout_of(int l) { return l == kLayers - 1 ? kHead : kHid; }
__host__ __device__ constexpr size_t layer_off(int l) {
    size_t off = 0;
    for (int k = 0; k < l; k++) off += size_t(cout_of(k)) * cin_of(k) * 9 + cout_of(k);
    return off;
}
__host__ __device__ constexpr size_t packed_off(int l) {  // bf16 elements
    size_t off = 0;
    for (int k = 0; k < l; k++) off += size_t(9) * cin_of(k) * cout_of(k);
    return off;
}
constexpr size_t kParams = layer_off(kLayers);
constexpr size_t kPacked = packed_off(kLayers);

constexpr uint64_t kWaitNs = 1000000000ull;  // 1 s

// Row-streaming convolution (k_sg_rows below): a CTA computes strips of RM
// output pixels of a run of rows; an input row of a strip is RW pixels.
constexpr int RM = 128, RW = RM + 2;
// Ring sizes of a layer's pipeline: accumulator rows in tensor memory (as
// pairs of adjacent rows) and shared-memory stages of two input rows.
template <int SLOTS, int STAGES>
struct Ring {
    static constexpr int slots = SLOTS, pairs = SLOTS / 2, stages = STAGES;
};
// One layer a CTA, two CTAs an SM: 256 tensor-memory columns a ring, so 8
// rows of 32 channels or 16 rows of 16 (the head; a longer ring splits the
// MMAs of fewer rows at its end).
template <int COUT>
using Ring1 = Ring<256 / COUT, 4>;
constexpr int kRowStages = 4;
constexpr int kRowGroups = 4;                 // epilogue groups of four warps (128 lanes)
constexpr int kRowEpiWarps = 4 * kRowGroups;
constexpr int kRowProducerWarp = kRowEpiWarps, kRowMmaWarp = kRowEpiWarps + 1;
constexpr int kRowThreads = 32 * (kRowEpiWarps + 2);

// Instruction descriptor of an M = RM, N = n MMA, kind::f16: f32 accumulator
// (bits 4-5 = 1), A and B bf16 (bits 7-9, 10-12 = 1), both K-major, N >> 3
// at bit 17, M >> 4 at bit 24.
__host__ __device__ constexpr uint32_t row_idesc(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(n >> 3) << 17) | (uint32_t(RM >> 4) << 24);
}

// Input rows of CIN channels in shared memory: per row, CIN / 8 chunk
// planes of RW 16-byte pixels; two rows a stage.
template <int CIN>
struct RowIn {
    static constexpr int C8 = CIN / 8, H2 = CIN / 16;
    static constexpr int PLANE = RW * 16;   // bytes per chunk plane of an input row
    static constexpr int ROW = C8 * PLANE;  // bytes per input row
    static constexpr int STAGE = (2 * ROW + 127) & ~127;
};

template <int CIN, int COUT>
struct RowCfg : RowIn<CIN> {
    using RowIn<CIN>::H2;
    static constexpr int NB = 3 * COUT;                // N of a full MMA: the three kernel rows stacked
    static constexpr int W_BYTES = 3 * H2 * 2 * NB * 16;  // = 9 x CIN x COUT bf16
    static constexpr uint32_t TMEM_COLS = Ring1<COUT>::slots * COUT;  // one layer a CTA
    static_assert(CIN % 16 == 0 && COUT % 16 == 0 && NB <= 256, "tcgen05 shape");
    static_assert(TMEM_COLS >= 32 && (TMEM_COLS & (TMEM_COLS - 1)) == 0, "tensor memory allocation");
};

// The develop output written by the head's epilogue (inference): picture
// pixels from network-frame quads.
struct RgbOut {
    const float* base;  // [3][hq][wq], network frame: each quad's colour
    int w, h;           // picture
    int rr, rc;         // mirrors of the network frame
    int has_matrix;
    float m[9];
    int layout;
    float* r;
    float* g;
    float* b;
    const unsigned* fallback;  // per 32x32 picture tile: developed by the plain kernel instead
    int tiles_x;
};

// Epilogue modes of the convolution.
enum : int { kHidden = 0, kHeadF32 = 1, kHeadRgb = 2 };

struct ConvArgs {
    const uint4* x;     // bf16 chunks [image][CIN/8][H][W]
    const uint4* w;     // the layer's packed weights (k_sg_pack_weights)
    const float* bias;  // [COUT]
    uint4* y;           // hidden layers: bf16 chunks [image][COUT/8][H][W]
    float* yf;          // head: f32 [image][16][H][W]
    const int4* valid;  // per image: x0, y0, x1, y1 (null: the whole image)
    int H, W;
    unsigned* error;    // bit 0: a tensor-core wait ran out of time
};

// --- tcgen05 / mbarrier helpers ------------------------------------------------

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor, no swizzle: start address, leading byte
// offset (between the two 8-element K chunks), stride byte offset (between
// 8-row groups of M or N), descriptor version 1 at bit 46.
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return uint64_t((addr & 0x3FFFFu) >> 4) | (uint64_t((lbo >> 4) & 0x3FFFu) << 16) |
           (uint64_t((sbo >> 4) & 0x3FFFu) << 32) | (uint64_t(1) << 46);
}

// The MMA and its commit are executed by a whole converged warp, which
// computes the (warp-uniform) addresses and descriptors; one lane, elected
// in each instruction, issues it.
__device__ __forceinline__ void umma_f16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p, e;\n\t"
        "elect.sync _|e, 0xffffffff;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "@e tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void umma_commit(uint32_t mbar) {
    asm volatile(
        "{\n\t.reg .pred e;\n\t"
        "elect.sync _|e, 0xffffffff;\n\t"
        "@e tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n\t}\n" ::"r"(mbar)
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t mbar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    return done != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Wait for phase `parity` of the mbarrier, for at most ~limit_ns and a fixed
// number of polls.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity, uint64_t limit_ns) {
    if (mbar_try_wait(mbar, parity)) return true;
    const uint64_t t0 = global_ns();
    for (uint32_t i = 0; i < (1u << 24); i++) {
        if (mbar_try_wait(mbar, parity)) return true;
        __nanosleep(64);
        if (global_ns() - t0 > limit_ns) return false;
    }
    return false;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

#define SG_R8(i) "=r"(v[i + 0]), "=r"(v[i + 1]), "=r"(v[i + 2]), "=r"(v[i + 3]), "=r"(v[i + 4]), \
                 "=r"(v[i + 5]), "=r"(v[i + 6]), "=r"(v[i + 7])

// 32 lanes x N f32 columns of tensor memory into registers (lane = thread).
template <int N>
__device__ __forceinline__ void tmem_load(uint32_t taddr, uint32_t* v);
template <>
__device__ __forceinline__ void tmem_load<32>(uint32_t taddr, uint32_t* v) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : SG_R8(0), SG_R8(8), SG_R8(16), SG_R8(24)
        : "r"(taddr));
}
template <>
__device__ __forceinline__ void tmem_load<16>(uint32_t taddr, uint32_t* v) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15}, [%16];"
        : SG_R8(0), SG_R8(8)
        : "r"(taddr));
}
#undef SG_R8

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
    const __nv_bfloat16 a = __float2bfloat16_rn(lo), b = __float2bfloat16_rn(hi);
    return uint32_t(__bfloat16_as_ushort(a)) | (uint32_t(__bfloat16_as_ushort(b)) << 16);
}

__device__ __forceinline__ float bf16_lo(uint32_t w) { return __uint_as_float(w << 16); }
__device__ __forceinline__ float bf16_hi(uint32_t w) { return __uint_as_float(w & 0xFFFF0000u); }

__device__ __forceinline__ bool in_valid(const int4* valid, int b, int x, int y) {
    if (!valid) return true;
    const int4 v = valid[b];
    return x >= v.x && y >= v.y && x < v.z && y < v.w;
}

// --- the convolution on the tensor cores --------------------------------------
//
// Row-streaming and warp-specialized. A work unit is a strip of RM = 128
// output pixels (columns sx0 .. sx0 + 127) over a run of rows; a persistent
// CTA takes units u = blockIdx.x, + gridDim.x, ... and walks each unit's
// input rows top to bottom, two at a time (a step):
//  - a producer warp: the layer's weights once (bulk copy), then a step's two
//    input rows (RW = 130 pixels each: one to the left and right of the
//    strip, every chunk) by one bulk copy per row and chunk plane into a ring
//    of stages, zeros written in place of the pixels outside the picture;
//  - an MMA warp (converged: it computes the descriptors as warp-uniform
//    values, an elected lane issues): per input row y, for each column offset
//    kx and 16-channel half, one tcgen05.mma with M = 128 (the strip's
//    pixels; A is the row shifted by kx), K = 16 and N = 3 x COUT: B stacks
//    the weights of kernel rows ky = 2, 1, 0, and the accumulator columns of
//    output rows y - 1, y, y + 1 are three consecutive slots of a ring in
//    tensor memory (two MMAs where the three slots wrap around the ring), so
//    each window byte read serves three output rows. Output rows pair up
//    (the slots of a pair are adjacent); a pair is complete after the step
//    that follows the one that opened it, and a commit hands it to the
//    epilogue;
//  - sixteen epilogue warps in four groups of four, a group per pair slot:
//    a warp reads its 32 lanes (pixels) of both rows with tcgen05.ld, writes
//    zeros back with tcgen05.st (the MMAs accumulate onto them), hands the
//    pair back, and adds the bias, applies ReLU and stores bf16 chunks (or the
//    f32 head, or the develop output).
// One wait and one commit per two rows keep the MMA warp issuing: an SM
// takes one tcgen05.mma about every 60 cycles, so these M = 128, N = 96
// products (48 cycles of tensor work each) leave it little time for anything
// else. Stages and pairs are passed by mbarriers (full/empty rings). Every
// wait is bounded; a wait that runs out sets the error flag and makes every
// role stop at its next step.

struct RowUnit {
    int img, sx0, sy0, rows;
};

__device__ __forceinline__ RowUnit row_unit(int u, int strips, int segs, int seg_rows, int strip_w, int H) {
    const int per = strips * segs;
    RowUnit r;
    r.img = u / per;
    const int k = u - r.img * per;
    r.sy0 = (k / strips) * seg_rows;
    r.sx0 = (k % strips) * strip_w;
    r.rows = min(seg_rows, H - r.sy0);
    return r;
}

// A unit's steps (input rows 0 .. rows + 1, two a step) and the output rows
// it takes in the ring (rounded up to pairs).
__device__ __forceinline__ int unit_steps(int rows) { return (rows + 3) / 2; }
__device__ __forceinline__ int unit_ring_rows(int rows) { return (rows + 1) & ~1; }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%1], %0;" ::"r"(bytes), "r"(bar) : "memory");
}

// Contiguous global -> shared bulk copy (16-byte aligned, size a multiple of 16).
__device__ __forceinline__ void bulk_copy(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

__device__ __forceinline__ void st_shared_zero16(uint32_t addr) {
    asm volatile("st.shared.v4.u32 [%0], {%1, %1, %1, %1};" ::"r"(addr), "r"(0u) : "memory");
}

// Zeros into 32 lanes x N f32 columns of tensor memory.
template <int N>
__device__ __forceinline__ void tmem_zero(uint32_t taddr);
template <>
__device__ __forceinline__ void tmem_zero<32>(uint32_t taddr) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, "
        "%1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1};" ::"r"(taddr),
        "r"(0u)
        : "memory");
}
template <>
__device__ __forceinline__ void tmem_zero<16>(uint32_t taddr) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, "
        "%1};" ::"r"(taddr),
        "r"(0u)
        : "memory");
}

// One thread's view, issued by the whole MMA warp: the MMAs of input row
// `row` (a stage's row) into blocks jlo .. jhi of the stacked N (block j:
// output row y - 1 + j, kernel row ky = 2 - j), block jlo's slot s0 (a block
// past the ring's end continues at slot 0). The descriptors differ from the
// row's and the weights' base descriptors only in the start address (bits
// 0-13, 16-byte units, no carry: shared addresses stay below 256 KB).
template <int CIN, int COUT, class R>
__device__ __forceinline__ void issue_row(uint32_t row, uint32_t w, uint32_t tmem, int s0, int jlo, int jhi) {
    using C = RowCfg<CIN, COUT>;
    const int nblk = jhi - jlo + 1, n1 = min(nblk, R::slots - s0);
    // A: row m = pixel sx0 - 1 + m + kx, 8-pixel groups 128 bytes apart, the
    // second K chunk the next chunk plane. B: [kx][half][K chunk][N][8].
    const uint64_t a0 = sdesc(row, C::PLANE, 128), b0 = sdesc(w, C::NB * 16, 128) + (uint32_t(jlo * COUT * 16) >> 4);
#pragma unroll
    for (int kx = 0; kx < 3; kx++) {
#pragma unroll
        for (int h = 0; h < C::H2; h++) {
            const uint64_t ad = a0 + (uint32_t(2 * h * C::PLANE + kx * 16) >> 4);
            const uint64_t bd = b0 + (uint32_t((kx * C::H2 + h) * 2 * C::NB * 16) >> 4);
            umma_f16(tmem + uint32_t(s0 * COUT), ad, bd, row_idesc(n1 * COUT), 1u);
            if (n1 < nblk) umma_f16(tmem, ad, bd + (uint32_t(n1 * COUT * 16) >> 4), row_idesc((nblk - n1) * COUT), 1u);
        }
    }
}

// Head channel c * 4 + 2 sy + sx of network quad (i, j), plus the quad's
// colour, is network pixel (2 i + sx, 2 j + sy), mirrored back to the
// picture; min(., 1), the matrix (src/demosaic.rs:700-720 for its operation
// order), and the store.
__device__ __forceinline__ void rgb_quad(const RgbOut& o, int i, int j, int wq, int hq, const float* hv) {
    const size_t plane = size_t(wq) * hq, q = size_t(j) * wq + i;
    const float b0 = o.base[q], b1 = o.base[plane + q], b2 = o.base[2 * plane + q];
    const int X0 = o.rc ? o.w - 1 - 2 * i : 2 * i, Y0 = o.rr ? o.h - 1 - 2 * j : 2 * j;
    if (o.fallback && o.fallback[(Y0 / kDevelopTile) * o.tiles_x + X0 / kDevelopTile]) return;
#pragma unroll
    for (int sy = 0; sy < 2; sy++)
#pragma unroll
        for (int sx = 0; sx < 2; sx++) {
            const int X = o.rc ? X0 - sx : X0 + sx, Y = o.rr ? Y0 - sy : Y0 + sy;
            if (X < 0 || Y < 0 || X >= o.w || Y >= o.h) continue;
            const int sidx = sy * 2 + sx;
            float r = fminf(__fadd_rn(hv[0 + sidx], b0), 1.0f);
            float g = fminf(__fadd_rn(hv[4 + sidx], b1), 1.0f);
            float b = fminf(__fadd_rn(hv[8 + sidx], b2), 1.0f);
            if (o.has_matrix) {
                const float r0 = r, g0 = g, bb0 = b;
                r = __fmaf_rn(bb0, o.m[2], __fmaf_rn(r0, o.m[0], __fmul_rn(g0, o.m[1])));
                g = __fmaf_rn(bb0, o.m[5], __fmaf_rn(r0, o.m[3], __fmul_rn(g0, o.m[4])));
                b = __fmaf_rn(bb0, o.m[8], __fmaf_rn(r0, o.m[6], __fmul_rn(g0, o.m[7])));
            }
            const size_t pi = size_t(Y) * o.w + X;
            if (o.layout == PRR_PLANAR) {
                o.r[pi] = r;
                o.g[pi] = g;
                o.b[pi] = b;
            } else {
                o.r[3 * pi] = r;
                o.r[3 * pi + 1] = g;
                o.r[3 * pi + 2] = b;
            }
        }
}

// One output pixel from its accumulator values v: bias, then ReLU and bf16
// chunks (hidden), the f32 head, or the develop output.
template <int COUT, int MODE>
__device__ __forceinline__ void store_pixel(const ConvArgs& a, const RgbOut& o, int img, int px, int py,
                                            const uint32_t* v, const float* bias) {
    const bool keep = in_valid(a.valid, img, px, py);
    if (MODE == kHeadRgb) {
        float hv[COUT];
#pragma unroll
        for (int c = 0; c < COUT; c++) hv[c] = __fadd_rn(__uint_as_float(v[c]), bias[c]);
        rgb_quad(o, px, py, a.W, a.H, hv);
    } else if (MODE == kHeadF32) {
        float* of = a.yf + (size_t(img) * kHead * a.H + py) * a.W + px;
#pragma unroll
        for (int c = 0; c < COUT; c++)
            of[size_t(c) * a.H * a.W] = keep ? __fadd_rn(__uint_as_float(v[c]), bias[c]) : 0.0f;
    } else {
        uint4* oy = a.y + (size_t(img) * (COUT / 8) * a.H + py) * a.W + px;
#pragma unroll
        for (int c8 = 0; c8 < COUT / 8; c8++) {
            float f[8];
#pragma unroll
            for (int e = 0; e < 8; e++) {
                const float s = __fadd_rn(__uint_as_float(v[c8 * 8 + e]), bias[c8 * 8 + e]);
                f[e] = keep ? fmaxf(s, 0.0f) : 0.0f;
            }
            oy[size_t(c8) * a.H * a.W] = make_uint4(pack_bf16x2(f[0], f[1]), pack_bf16x2(f[2], f[3]),
                                                    pack_bf16x2(f[4], f[5]), pack_bf16x2(f[6], f[7]));
        }
    }
}

// The input rows of a unit as one pipeline reads them: rows y0 .. y0 + nin - 1
// (those inside the picture), window column c = pixel xw + c, two rows a
// stage.
struct RowSpan {
    int img, xw, y0, nin;
};

// Producer warp: the span's rows into the stage ring, one bulk copy per row
// and chunk plane, zeros in place of the pixels outside the picture. False
// when a wait ran out.
template <int CIN, class R>
__device__ __forceinline__ bool produce_span(const ConvArgs& a, const RowSpan& sp, uint32_t st0, uint32_t sfull0,
                                             uint32_t sempty0, int& filled, volatile int& aborted, int lane) {
    using I = RowIn<CIN>;
    const int xa = max(sp.xw, 0), xb = min(sp.xw + RW, a.W);
    const int zl = xa - sp.xw, zr = sp.xw + RW - xb, nz = zl + zr;
    const uint32_t row_bytes = uint32_t(xb - xa) * 16;
    for (int t = 0; 2 * t < sp.nin; t++) {
        const int s = filled % R::stages;
        // The stage is free once the MMAs of fill filled - R::stages are done
        // (the first round passes: its parity refers to the phase before the
        // barrier's first).
        int got = 1;
        if (lane == 0) got = !aborted && mbar_wait(sempty0 + 8 * s, uint32_t(((filled / R::stages) & 1) ^ 1), kWaitNs);
        if (!__shfl_sync(0xFFFFFFFFu, got, 0)) return false;
        const uint32_t dst = st0 + uint32_t(s * I::STAGE);
        bool in[2];
#pragma unroll
        for (int e = 0; e < 2; e++) {
            const int i = 2 * t + e, y = sp.y0 + i;
            in[e] = i < sp.nin && y >= 0 && y < a.H;
        }
        if (nz > 0 && (in[0] || in[1])) {
            for (int e = 0; e < 2; e++) {
                if (!in[e]) continue;
                for (int z = lane; z < I::C8 * nz; z += 32) {
                    const int p = z / nz, c = z - p * nz;
                    st_shared_zero16(dst + uint32_t(e * I::ROW + p * I::PLANE + (c < zl ? c : RW - nz + c) * 16));
                }
            }
            // The zeros are read by the tensor cores (the async proxy).
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        }
        __syncwarp();
        if (lane == 0) {
            const uint32_t bytes = uint32_t(I::C8) * row_bytes * uint32_t(int(in[0]) + int(in[1]));
            if (bytes == 0) {
                mbar_arrive(sfull0 + 8 * s);
            } else {
                mbar_expect_tx(sfull0 + 8 * s, bytes);
                for (int e = 0; e < 2; e++) {
                    if (!in[e]) continue;
                    const uint4* src = a.x + (size_t(sp.img) * I::C8 * a.H + (sp.y0 + 2 * t + e)) * a.W + xa;
                    for (int p = 0; p < I::C8; p++)
                        bulk_copy(dst + uint32_t(e * I::ROW + p * I::PLANE + zl * 16), src + size_t(p) * a.H * a.W,
                                  row_bytes, sfull0 + 8 * s);
                }
            }
        }
        filled++;
    }
    return true;
}

// Barriers of one layer's pipeline: its input stages (full / empty) and its
// accumulator pairs (full / empty), R::stages and R::pairs of each.
struct RowBars {
    uint32_t sfull, sempty, ofull, oempty;
};

// MMA warp (converged; an elected lane issues): one unit of one layer, output
// rows 0 .. rows - 1 (ring rows kb ..), input row i = row y0 + i of the
// picture (rows outside it give nothing), read from stage ring st0 with
// stages stage_bytes apart. False when a wait ran out.
template <int CIN, int COUT, class R>
__device__ __forceinline__ bool mma_unit(int rows, int y0, int H, uint32_t st0, int stage_bytes, const RowBars& b,
                                         uint32_t w, uint32_t tmem, int& kb, int& used, volatile int& aborted) {
    using C = RowCfg<CIN, COUT>;
    for (int t = 0; t < unit_steps(rows); t++) {
        if (2 * t < rows) {
            // The step opens output rows 2t, 2t + 1: their pair must be
            // drained and zeroed (phase u of use u).
            const int P = kb / 2 + t;
            if (!__all_sync(0xFFFFFFFFu, !aborted && mbar_wait(b.oempty + 8 * (P % R::pairs),
                                                               uint32_t((P / R::pairs) & 1), kWaitNs)))
                return false;
        }
        const int s = used % R::stages;
        if (!__all_sync(0xFFFFFFFFu, !aborted && mbar_wait(b.sfull + 8 * s, uint32_t((used / R::stages) & 1), kWaitNs)))
            return false;
        tc_fence_after();
#pragma unroll
        for (int e = 0; e < 2; e++) {
            const int i = 2 * t + e, y = y0 + i;
            if (i > rows + 1 || y < 0 || y >= H) continue;
            // Blocks j of output rows i - 2 + j inside the unit.
            const int jlo = max(0, 2 - i), jhi = min(2, rows + 1 - i);
            issue_row<CIN, COUT, R>(st0 + uint32_t(s * stage_bytes + e * C::ROW), w, tmem, (kb + i - 2 + jlo) % R::slots,
                                    jlo, jhi);
        }
        umma_commit(b.sempty + 8 * s);  // the stage, once these MMAs have read it
        used++;
        // Output rows 2t - 2, 2t - 1 took their last products (from input row
        // 2t + 1): hand the pair to the epilogue.
        if (t >= 1) umma_commit(b.ofull + 8 * ((kb / 2 + t - 1) % R::pairs));
    }
    kb += unit_ring_rows(rows);
    return true;
}

// Epilogue warp: wait for ring pair P (slot pair P % R::pairs) and read
// its first row; the caller reads the second with pair_second.
template <int COUT, class R>
__device__ __forceinline__ bool pair_first(const RowBars& b, int P, uint32_t slot0, uint32_t* v, volatile int& aborted) {
    bool got = !aborted && mbar_wait(b.ofull + 8 * (P % R::pairs), uint32_t((P / R::pairs) & 1), kWaitNs);
    if (!__all_sync(0xFFFFFFFFu, got)) return false;  // the warp-collective loads need one branch per warp
    tc_fence_after();
    tmem_load<COUT>(slot0, v);
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    tmem_zero<COUT>(slot0);  // the MMAs accumulate onto zeros
    return true;
}

// The pair's second row into v; the pair goes back to the MMA warp.
template <int COUT, class R>
__device__ __forceinline__ void pair_second(const RowBars& b, int P, uint32_t slot1, uint32_t* v, int lane) {
    tmem_load<COUT>(slot1, v);
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    tmem_zero<COUT>(slot1);
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
    tc_fence_before();
    __syncwarp();
    if (lane == 0) mbar_arrive(b.oempty + 8 * (P % R::pairs));
}

// The ring's pair slot g of a warp's lane quarter starts zeroed (phase 0 of
// the pair's empty barrier).
template <int COUT>
__device__ __forceinline__ void pair_init(const RowBars& b, int g, uint32_t slot0, int lane) {
    tmem_zero<COUT>(slot0);
    tmem_zero<COUT>(slot0 + uint32_t(COUT));
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
    tc_fence_before();
    __syncwarp();
    if (lane == 0) mbar_arrive(b.oempty + 8 * g);
}

template <class R>
__device__ __forceinline__ void init_bars(const RowBars& b, uint32_t full_count) {
    for (int s = 0; s < R::stages; s++) {
        mbar_init(b.sfull + 8 * s, full_count);  // the stage's producer arrival(s)
        mbar_init(b.sempty + 8 * s, 1);          // the MMA warp's commit
    }
    for (int q = 0; q < R::pairs; q++) {
        mbar_init(b.ofull + 8 * q, 1);   // the MMA warp's commit
        mbar_init(b.oempty + 8 * q, 4);  // the four warps of the pair's epilogue group
    }
}

// One layer (k_sg_rows): persistent CTAs, two an SM, in the roles above.
template <int CIN, int COUT, int MODE>
__global__ void __launch_bounds__(kRowThreads, 2) k_sg_rows(ConvArgs a, RgbOut o, int strips, int segs, int seg_rows,
                                                             int nunits) {
    using C = RowCfg<CIN, COUT>;
    using R = Ring1<COUT>;
    constexpr int S = R::stages, Q = R::pairs;
    static_assert(Q % kRowGroups == 0, "a pair slot belongs to one epilogue group");
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ __align__(8) uint64_t bars[2 * S + 2 * Q + 2];
    __shared__ uint32_t tmem_slot;
    __shared__ float bias_s[COUT];
    volatile __shared__ int aborted;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int first = blockIdx.x, stride = gridDim.x;
    const int n = first < nunits ? (nunits - 1 - first) / stride + 1 : 0;  // this CTA's units
    // Weights, then the stages, 128-byte aligned.
    const uint32_t wsm = smem_u32(smem);
    const uint32_t st0 = wsm + uint32_t((C::W_BYTES + 127) & ~127);
    auto bar = [&](int i) { return smem_u32(&bars[i]); };
    const RowBars rb{bar(0), bar(S), bar(2 * S), bar(2 * S + Q)};
    const uint32_t wbar = bar(2 * S + 2 * Q), dbar = wbar + 8;
    if (tid == 0) {
        init_bars<R>(rb, 1);
        mbar_init(wbar, 1);
        mbar_init(dbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        aborted = 0;
    }
    if (tid < COUT) bias_s[tid] = a.bias[tid];
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                     "r"(C::TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;
    int filled = 0;  // producer: stages filled
    bool ok = true;

    if (warp == kRowProducerWarp) {
        if (lane == 0) {
            mbar_expect_tx(wbar, uint32_t(C::W_BYTES));
            bulk_copy(wsm, a.w, uint32_t(C::W_BYTES), wbar);
        }
        for (int u = 0; ok && u < n; u++) {
            const RowUnit ru = row_unit(first + u * stride, strips, segs, seg_rows, RM, a.H);
            ok = produce_span<CIN, R>(a, RowSpan{ru.img, ru.sx0 - 1, ru.sy0 - 1, ru.rows + 2}, st0, rb.sfull, rb.sempty,
                                      filled, aborted, lane);
        }
    } else if (warp == kRowMmaWarp) {
        ok = __all_sync(0xFFFFFFFFu, mbar_wait(wbar, 0, kWaitNs));
        int kb = 0, used = 0;  // ring rows of the earlier units; stages consumed
        for (int u = 0; ok && u < n; u++) {
            const RowUnit ru = row_unit(first + u * stride, strips, segs, seg_rows, RM, a.H);
            ok = mma_unit<CIN, COUT, R>(ru.rows, ru.sy0 - 1, a.H, st0, C::STAGE, rb, wsm, tmem, kb, used, aborted);
        }
        umma_commit(dbar);  // every issued MMA
    } else {
        const int g = warp >> 2, q = warp & 3;  // group (pair slots g, g + kRowGroups, ...); lane quarter
        const uint32_t lanes = uint32_t(32 * q) << 16;
        for (int ps = g; ps < Q; ps += kRowGroups) pair_init<COUT>(rb, ps, tmem + lanes + uint32_t(2 * ps * COUT), lane);
        int kb = 0;
        for (int u = 0; ok && u < n; u++) {
            const RowUnit ru = row_unit(first + u * stride, strips, segs, seg_rows, RM, a.H);
            const int px = ru.sx0 + 32 * q + lane;
            for (int p = ((g - kb / 2) % kRowGroups + kRowGroups) % kRowGroups; 2 * p < ru.rows; p += kRowGroups) {
                const int P = kb / 2 + p;
                const uint32_t slot0 = tmem + lanes + uint32_t(2 * (P % Q) * COUT);
                uint32_t v[COUT];
                if (!(ok = pair_first<COUT, R>(rb, P, slot0, v, aborted))) break;
                if (px < a.W) store_pixel<COUT, MODE>(a, o, ru.img, px, ru.sy0 + 2 * p, v, bias_s);
                pair_second<COUT, R>(rb, P, slot0 + uint32_t(COUT), v, lane);
                if (px < a.W && 2 * p + 1 < ru.rows) store_pixel<COUT, MODE>(a, o, ru.img, px, ru.sy0 + 2 * p + 1, v, bias_s);
            }
            kb += unit_ring_rows(ru.rows);
        }
    }
    if (!ok && lane == 0) {
        if (!aborted) atomicOr(a.error, 1u);
        aborted = 1;
    }
    __syncthreads();
    if (aborted && warp == kRowMmaWarp) mbar_wait(dbar, 0, kWaitNs);  // issued MMAs finish (bounded)
    if (aborted && tid == kRowProducerWarp * 32) {
        // Let the issued copies land (bounded) before the CTA exits: the last
        // fill of each stage is its latest phase.
        for (int j = max(0, filled - S); j < filled; j++)
            mbar_wait(rb.sfull + 8 * (j % S), uint32_t((j / S) & 1), kWaitNs / 8);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(C::TMEM_COLS));
}

// Two layers in one pass: layer A (CIN -> 32) feeds layer B (32 -> COUT)
// through a ring of row stages in shared memory, so A's output never goes
// to HBM. A's MMA warp and epilogue run the one-layer scheme over A's rows
// (output rows sy0 - 1 .. sy0 + rows, the ones B reads); A's epilogue writes
// each finished pair of rows, biased and rectified as bf16 chunks (zeros
// outside the picture), into a stage of the ring, which B's MMA warp reads as
// its input rows. A's strip is 128 pixels from sx0 - 1, so B's outputs are
// exact for the 126 pixels from sx0 (lanes 126, 127 lack their right
// neighbours and are not stored): strips are RM - 2 pixels apart.
// Warps: 0-3 A's epilogue, 4-7 B's epilogue, the producer, A's MMA warp,
// B's MMA warp. Two CTAs an SM (Ring2: each layer's ring takes 4 x 32
// tensor-memory columns, and a CTA about 100 KB of shared memory), so that
// one CTA's MMAs are issued while the other's warps wait.
using Ring2 = Ring<4, 2>;
constexpr int kFuseEpiB = 4, kFuseProducerWarp = 8, kFuseMmaA = 9, kFuseMmaB = 10;  // A's epilogue: warps 0-3
constexpr int kFuseThreads = 32 * (kFuseMmaB + 1);
constexpr int kFuseStrip = RM - 2;

template <int CIN, int COUT>
struct FuseCfg {
    using A = RowCfg<CIN, kHid>;
    using B = RowCfg<kHid, COUT>;
    static constexpr int WA = (A::W_BYTES + 127) & ~127, WB = (B::W_BYTES + 127) & ~127;
    static constexpr int SMEM = WA + WB + Ring2::stages * (A::STAGE + B::STAGE);
    static constexpr uint32_t TMEM_B = Ring2::slots * kHid;  // B's ring after A's
    static constexpr uint32_t TMEM_COLS = 256;
    static_assert(TMEM_B + Ring2::slots * COUT <= TMEM_COLS, "tensor memory");
};

template <int CIN, int COUT, int MODE>
__global__ void __launch_bounds__(kFuseThreads, 2) k_sg_rows2(ConvArgs a, ConvArgs bl, RgbOut o, int strips, int segs,
                                                              int seg_rows, int nunits) {
    using F = FuseCfg<CIN, COUT>;
    using LA = typename F::A;
    using LB = typename F::B;
    using R = Ring2;
    constexpr int S = R::stages, Q = R::pairs;
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ __align__(8) uint64_t bars[4 * S + 4 * Q + 3];
    __shared__ uint32_t tmem_slot;
    __shared__ float bias_a[kHid], bias_b[COUT];
    volatile __shared__ int aborted;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int first = blockIdx.x, stride = gridDim.x;
    const int n = first < nunits ? (nunits - 1 - first) / stride + 1 : 0;  // this CTA's units
    // A's weights, B's weights, A's input stages, the middle ring.
    const uint32_t wa = smem_u32(smem), wb = wa + uint32_t(F::WA), sta = wb + uint32_t(F::WB),
                   mid = sta + uint32_t(S * LA::STAGE);
    auto bar = [&](int i) { return smem_u32(&bars[i]); };
    const RowBars ra{bar(0), bar(S), bar(2 * S), bar(2 * S + Q)};
    const RowBars rb{bar(2 * S + 2 * Q), bar(3 * S + 2 * Q), bar(4 * S + 2 * Q), bar(4 * S + 3 * Q)};
    const uint32_t wbar = bar(4 * S + 4 * Q), dbar_a = wbar + 8, dbar_b = wbar + 16;
    if (tid == 0) {
        init_bars<R>(ra, 1);
        init_bars<R>(rb, 4);  // the middle ring's stages: A's four epilogue warps
        mbar_init(wbar, 1);
        mbar_init(dbar_a, 1);
        mbar_init(dbar_b, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        aborted = 0;
    }
    if (tid < kHid) bias_a[tid] = a.bias[tid];
    if (tid < COUT) bias_b[tid] = bl.bias[tid];
    // Middle-ring window columns 128 and 129 (right of A's 128 pixels) stay
    // zero: they reach only B's lanes 126 and 127, which are not stored.
    for (int z = tid; z < S * 2 * LB::C8 * 2; z += blockDim.x) {
        const int c = z & 1, p = (z >> 1) % LB::C8, e = (z / (2 * LB::C8)) & 1, s = z / (4 * LB::C8);
        st_shared_zero16(mid + uint32_t(s * LB::STAGE + e * LB::ROW + p * LB::PLANE + (RM + c) * 16));
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                     "r"(F::TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;
    int filled = 0;  // producer: stages filled
    bool ok = true;

    if (warp == kFuseProducerWarp) {
        if (lane == 0) {
            mbar_expect_tx(wbar, uint32_t(LA::W_BYTES + LB::W_BYTES));
            bulk_copy(wa, a.w, uint32_t(LA::W_BYTES), wbar);
            bulk_copy(wb, bl.w, uint32_t(LB::W_BYTES), wbar);
        }
        for (int u = 0; ok && u < n; u++) {
            const RowUnit ru = row_unit(first + u * stride, strips, segs, seg_rows, kFuseStrip, a.H);
            ok = produce_span<CIN, R>(a, RowSpan{ru.img, ru.sx0 - 2, ru.sy0 - 2, ru.rows + 4}, sta, ra.sfull,
                                      ra.sempty, filled, aborted, lane);
        }
    } else if (warp == kFuseMmaA || warp == kFuseMmaB) {
        const bool is_a = warp == kFuseMmaA;
        ok = __all_sync(0xFFFFFFFFu, mbar_wait(wbar, 0, kWaitNs));
        int kb = 0, used = 0;
        for (int u = 0; ok && u < n; u++) {
            const RowUnit ru = row_unit(first + u * stride, strips, segs, seg_rows, kFuseStrip, a.H);
            ok = is_a ? mma_unit<CIN, kHid, R>(ru.rows + 2, ru.sy0 - 2, a.H, sta, LA::STAGE, ra, wa, tmem, kb, used,
                                               aborted)
                      : mma_unit<kHid, COUT, R>(ru.rows, ru.sy0 - 1, a.H, mid, LB::STAGE, rb, wb, tmem + F::TMEM_B, kb,
                                                used, aborted);
        }
        umma_commit(is_a ? dbar_a : dbar_b);  // every issued MMA
    } else if (warp < kFuseEpiB) {
        // A's epilogue: pairs of A's output rows into the middle ring.
        const int q = warp & 3, m = 32 * q + lane;
        const uint32_t lanes = uint32_t(32 * q) << 16;
        for (int ps = 0; ps < Q; ps++) pair_init<kHid>(ra, ps, tmem + lanes + uint32_t(2 * ps * kHid), lane);
        int kb = 0;
        for (int u = 0; ok && u < n; u++) {
            const RowUnit ru = row_unit(first + u * stride, strips, segs, seg_rows, kFuseStrip, a.H);
            const int rows_a = ru.rows + 2, px = ru.sx0 - 1 + m;
            for (int p = 0; 2 * p < rows_a; p++) {
                const int P = kb / 2 + p, ms = P % S;
                const uint32_t slot0 = tmem + lanes + uint32_t(2 * (P % Q) * kHid);
                // The middle stage must have been read by B's MMAs (the first
                // round passes: its parity refers to the phase before the
                // barrier's first).
                ok = __all_sync(0xFFFFFFFFu,
                                !aborted && mbar_wait(rb.sempty + 8 * ms, uint32_t(((P / S) & 1) ^ 1), kWaitNs));
                if (!ok) break;
                uint32_t v[kHid];
                if (!(ok = pair_first<kHid, R>(ra, P, slot0, v, aborted))) break;
                const uint32_t dst = mid + uint32_t(ms * LB::STAGE + m * 16);
#pragma unroll 1
                for (int e = 0; e < 2; e++) {
                    if (e == 1) pair_second<kHid, R>(ra, P, slot0 + uint32_t(kHid), v, lane);
                    const int y = ru.sy0 - 1 + 2 * p + e;
                    const bool keep = px >= 0 && px < a.W && y >= 0 && y < a.H && in_valid(a.valid, ru.img, px, y);
#pragma unroll
                    for (int c8 = 0; c8 < kHid / 8; c8++) {
                        float f[8];
#pragma unroll
                        for (int k = 0; k < 8; k++) {
                            const float s = __fadd_rn(__uint_as_float(v[c8 * 8 + k]), bias_a[c8 * 8 + k]);
                            f[k] = keep ? fmaxf(s, 0.0f) : 0.0f;
                        }
                        asm volatile("st.shared.v4.u32 [%0], {%1, %2, %3, %4};" ::"r"(
                                         dst + uint32_t(e * LB::ROW + c8 * LB::PLANE)),
                                     "r"(pack_bf16x2(f[0], f[1])), "r"(pack_bf16x2(f[2], f[3])),
                                     "r"(pack_bf16x2(f[4], f[5])), "r"(pack_bf16x2(f[6], f[7]))
                                     : "memory");
                    }
                }
                // B's MMAs read the stage through the async proxy.
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                __syncwarp();
                if (lane == 0) mbar_arrive(rb.sfull + 8 * ms);
            }
            kb += unit_ring_rows(rows_a);
        }
    } else {
        // B's epilogue: pairs of B's output rows to memory.
        const int q = warp & 3, m = 32 * q + lane;
        const uint32_t lanes = uint32_t(32 * q) << 16;
        for (int ps = 0; ps < Q; ps++) pair_init<COUT>(rb, ps, tmem + F::TMEM_B + lanes + uint32_t(2 * ps * COUT), lane);
        int kb = 0;
        for (int u = 0; ok && u < n; u++) {
            const RowUnit ru = row_unit(first + u * stride, strips, segs, seg_rows, kFuseStrip, a.H);
            const int px = ru.sx0 + m;
            const bool store = m < kFuseStrip && px < a.W;
            for (int p = 0; 2 * p < ru.rows; p++) {
                const int P = kb / 2 + p;
                const uint32_t slot0 = tmem + F::TMEM_B + lanes + uint32_t(2 * (P % Q) * COUT);
                uint32_t v[COUT];
                if (!(ok = pair_first<COUT, R>(rb, P, slot0, v, aborted))) break;
                if (store) store_pixel<COUT, MODE>(bl, o, ru.img, px, ru.sy0 + 2 * p, v, bias_b);
                pair_second<COUT, R>(rb, P, slot0 + uint32_t(COUT), v, lane);
                if (store && 2 * p + 1 < ru.rows) store_pixel<COUT, MODE>(bl, o, ru.img, px, ru.sy0 + 2 * p + 1, v, bias_b);
            }
            kb += unit_ring_rows(ru.rows);
        }
    }
    if (!ok && lane == 0) {
        if (!aborted) atomicOr(a.error, 1u);
        aborted = 1;
    }
    __syncthreads();
    if (aborted && (warp == kFuseMmaA || warp == kFuseMmaB))
        mbar_wait(warp == kFuseMmaA ? dbar_a : dbar_b, 0, kWaitNs);  // issued MMAs finish (bounded)
    if (aborted && tid == kFuseProducerWarp * 32) {
        for (int j = max(0, filled - S); j < filled; j++)
            mbar_wait(ra.sfull + 8 * (j % S), uint32_t((j / S) & 1), kWaitNs / 8);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(F::TMEM_COLS));
}

// cuTensorMapEncodeTiled, looked up once through the runtime (no link
// against the driver library).
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// The driver's encoder, looked up once (a thread-safe static initializer);
// null when the runtime cannot find it.
EncodeTiledFn encode_tiled() {
    static const EncodeTiledFn fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        const cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q);
        return e == cudaSuccess && q == cudaDriverEntryPointSuccess ? reinterpret_cast<EncodeTiledFn>(p) : nullptr;
    }();
    return fn;
}

// Rows per work unit: the run length whose units, spread over `ctas` CTAs,
// give the fewest input rows to the busiest CTA (a unit of S rows reads
// S + halo; a CTA's rows follow one another through its pipeline, so a CTA,
// not an SM, sets the pace).
int row_segment(int strips, int H, int images, long ctas, int halo) {
    int best = H;
    long best_cost = LONG_MAX;
    for (int S = 8;; S += 8) {
        const int rows = std::min(S, H), segs = (H + rows - 1) / rows;
        const long units = long(strips) * segs * images;
        const long cost = (units + ctas - 1) / ctas * (rows + halo);
        if (cost < best_cost) {
            best_cost = cost;
            best = rows;
        }
        if (S >= H) break;
    }
    return best;
}

// The SM count of the current device, and the kernel's shared-memory limit
// set once per device (kept per device in atomics: contexts on several
// threads launch too).
template <class K>
cudaError_t kernel_setup(K kernel, int smem, std::atomic<int>* sms_of, int* sms) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    *sms = sms_of[dev].load(std::memory_order_acquire);
    if (*sms == 0) {
        e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return e;
        sms_of[dev].store(*sms, std::memory_order_release);
    }
    return cudaSuccess;
}

template <int CIN, int COUT, int MODE>
cudaError_t conv_launch(const ConvArgs& a, const RgbOut& o, int images, cudaStream_t s) {
    using C = RowCfg<CIN, COUT>;
    // Weights and the row stages; at least 80 KB, so that no more than two
    // CTAs share an SM (their accumulator rings fit in its 512 tensor-memory
    // columns; a third CTA's allocation would wait for one of them).
    constexpr int smem = std::max(((C::W_BYTES + 127) & ~127) + kRowStages * C::STAGE, 80 * 1024);
    static std::atomic<int> sms_of[kMaxDevices];
    int sms = 0;
    const cudaError_t e = kernel_setup(k_sg_rows<CIN, COUT, MODE>, smem, sms_of, &sms);
    if (e != cudaSuccess) return e;
    if (a.W <= 0 || a.H <= 0 || images <= 0) return cudaErrorInvalidValue;
    const int strips = (a.W + RM - 1) / RM;
    const int seg_rows = row_segment(strips, a.H, images, 2L * sms, 2);
    const int segs = (a.H + seg_rows - 1) / seg_rows;
    const long nunits = long(strips) * segs * images;
    if (nunits > INT_MAX) return cudaErrorInvalidValue;
    const int grid = int(std::max(1L, std::min(nunits, 2L * sms)));
    k_sg_rows<CIN, COUT, MODE><<<grid, kRowThreads, smem, s>>>(a, o, strips, segs, seg_rows, int(nunits));
    count_launch();
    return cudaGetLastError();
}

// Layers A (a: CIN -> 32) and B (b: 32 -> COUT) in one pass.
template <int CIN, int COUT, int MODE>
cudaError_t conv2_launch(const ConvArgs& a, const ConvArgs& b, const RgbOut& o, int images, cudaStream_t s) {
    constexpr int smem = FuseCfg<CIN, COUT>::SMEM;
    static_assert(smem <= 227 * 1024, "shared memory");
    static std::atomic<int> sms_of[kMaxDevices];
    int sms = 0;
    const cudaError_t e = kernel_setup(k_sg_rows2<CIN, COUT, MODE>, smem, sms_of, &sms);
    if (e != cudaSuccess) return e;
    if (a.W <= 0 || a.H <= 0 || images <= 0 || b.W != a.W || b.H != a.H) return cudaErrorInvalidValue;
    const int strips = (a.W + kFuseStrip - 1) / kFuseStrip;
    const int seg_rows = row_segment(strips, a.H, images, 2L * sms, 4);
    const int segs = (a.H + seg_rows - 1) / seg_rows;
    const long nunits = long(strips) * segs * images;
    if (nunits > INT_MAX) return cudaErrorInvalidValue;
    const int grid = int(std::max(1L, std::min(nunits, 2L * sms)));
    k_sg_rows2<CIN, COUT, MODE><<<grid, kFuseThreads, smem, s>>>(a, b, o, strips, segs, seg_rows, int(nunits));
    count_launch();
    return cudaGetLastError();
}

// --- input packing, weights, output ------------------------------------------------

struct PackArgs {
    const uint16_t* codes;
    uint32_t stride;
    int w, h, wq, hq;
    uint32_t c0[8], cd[8];
    int rr, rc, black;  // red sensel of a quad (row, column); the network frame mirrors by them
    float one_over_range, bs, wb0, wb1;
    float n0, n1, n2;
    uint4* in;      // [2][hq][wq] chunks
    float* base;    // [3][hq][wq]
    float* noise_minmax;  // optional: atomic min / max of the noise channel (as ordered ints)
    // Optional (the develop's fallback): per 32x32 picture tile, a nonzero
    // flag when a quad's noise channel leaves [fb_lo, fb_hi], and the count
    // of such tiles.
    unsigned* fb_flags;
    unsigned* fb_count;
    int tiles_x;
    float fb_lo, fb_hi;
};

__device__ __forceinline__ float sg_nrm(const PackArgs& p, int x, int y) {
    x = min(x, p.w - 1);
    y = min(y, p.h - 1);
    const uint32_t lin = curve_apply(p.c0, p.cd, p.codes[size_t(y) * p.stride + x]);
    return __fmul_rn(p.one_over_range, float(int32_t(lin) - p.black));
}

// Mean green of quad (i, j), the quad grid clamped at its edges.
__device__ __forceinline__ float sg_green(const PackArgs& p, int i, int j) {
    i = min(max(i, 0), p.wq - 1);
    j = min(max(j, 0), p.hq - 1);
    const float gr = sg_nrm(p, 2 * i + 1 - p.rc, 2 * j + p.rr);
    const float gb = sg_nrm(p, 2 * i + p.rc, 2 * j + 1 - p.rr);
    return __fmul_rn(__fadd_rn(gr, gb), 0.5f);
}

// Network-frame quad (i, j) is picture quad (i, j) mirrored horizontally
// when red sits in the right column of a quad and vertically when it sits in
// the bottom row, so that every Bayer pattern reaches the network as RGGB.
__host__ __device__ __forceinline__ int mirror_q(int i, int n, int flip) { return flip ? n - 1 - i : i; }

// A CTA packs a tile of kPackW x kPackH network-frame quads. Each quad's
// mean green is computed once into shared memory, with a one-quad halo
// (clamped at the picture's edges as sg_green clamps), for the neighbours'
// gradients and Laplacian.
constexpr int kPackW = 32, kPackH = 8;

__global__ void __launch_bounds__(kPackW * kPackH) k_sg_pack(PackArgs p) {
    __shared__ float gms[kPackH + 2][kPackW + 2];
    const int tx = threadIdx.x % kPackW, ty = threadIdx.x / kPackW;
    const int i0 = blockIdx.x * kPackW, j0 = blockIdx.y * kPackH;
    const int i = i0 + tx, j = j0 + ty;
    const bool inside = i < p.wq && j < p.hq;
    // Network-frame quad (i, j) is picture quad (si, sj).
    const int si = mirror_q(min(i, p.wq - 1), p.wq, p.rc), sj = mirror_q(min(j, p.hq - 1), p.hq, p.rr);
    const int x0 = 2 * si, y0 = 2 * sj;
    const float gr = sg_nrm(p, x0 + 1 - p.rc, y0 + p.rr);
    const float gb = sg_nrm(p, x0 + p.rc, y0 + 1 - p.rr);
    const float gm = __fmul_rn(__fadd_rn(gr, gb), 0.5f);
    gms[ty + 1][tx + 1] = gm;  // a quad past the picture's edge: its clamped neighbour, as sg_green
    // The halo ring: 2 (kPackW + 2) + 2 kPackH cells.
    for (int c = threadIdx.x; c < 2 * (kPackW + 2) + 2 * kPackH; c += blockDim.x) {
        int cx, cy;
        if (c < 2 * (kPackW + 2)) {
            cx = c % (kPackW + 2);
            cy = c < kPackW + 2 ? 0 : kPackH + 1;
        } else {
            const int k = c - 2 * (kPackW + 2);
            cx = (k & 1) ? kPackW + 1 : 0;
            cy = 1 + (k >> 1);
        }
        gms[cy][cx] = sg_green(p, mirror_q(i0 - 1 + cx, p.wq, p.rc), mirror_q(j0 - 1 + cy, p.hq, p.rr));
    }
    __syncthreads();
    if (!inside) return;
    const float r = __fmul_rn(sg_nrm(p, x0 + p.rc, y0 + p.rr), p.wb0);
    const float b = __fmul_rn(sg_nrm(p, x0 + 1 - p.rc, y0 + 1 - p.rr), p.wb1);
    const float t = __fadd_rn(p.bs, gm);
    const float var = __fadd_rn(p.n2, fmaxf(p.n1, __fmul_rn(p.n0, __fmul_rn(t, t))));
    const float noise = __fmul_rn(64.0f, __fsqrt_rn(var));
    // Network east / west / south / north neighbours.
    const float ge = gms[ty + 1][tx + 2], gw = gms[ty + 1][tx];
    const float gs = gms[ty + 2][tx + 1], gn = gms[ty][tx + 1];
    const float gx = __fmul_rn(__fsub_rn(ge, gw), 0.5f), gy = __fmul_rn(__fsub_rn(gs, gn), 0.5f);
    const float lap = __fsub_rn(gm, __fmul_rn(__fadd_rn(__fadd_rn(ge, gw), __fadd_rn(gs, gn)), 0.25f));
    auto d4 = [](float v, float ref) { return __fmul_rn(__fsub_rn(v, ref), 4.0f); };
    const size_t q = size_t(j) * p.wq + i, plane = size_t(p.wq) * p.hq;
    p.in[q] = make_uint4(pack_bf16x2(d4(r, gm), d4(gr, gm)), pack_bf16x2(d4(gb, gm), d4(b, gm)),
                         pack_bf16x2(noise, gm), pack_bf16x2(__fmul_rn(gx, 4.0f), __fmul_rn(gy, 4.0f)));
    p.in[plane + q] = make_uint4(pack_bf16x2(__fmul_rn(lap, 4.0f), 0.0f), 0u, 0u, 0u);
    p.base[q] = r;
    p.base[plane + q] = gm;
    p.base[2 * plane + q] = b;
    // The noise channel as the network sees it (bf16).
    const float nb = bf16_lo(pack_bf16x2(noise, 0.0f));
    if (p.noise_minmax) {
        // As a non-negative float, its bits order like ints.
        atomicMin(reinterpret_cast<int*>(p.noise_minmax), __float_as_int(nb));
        atomicMax(reinterpret_cast<int*>(p.noise_minmax) + 1, __float_as_int(nb));
    }
    if (p.fb_flags && !(nb >= p.fb_lo && nb <= p.fb_hi)) {
        const int tile = (sj / (kDevelopTile / 2)) * p.tiles_x + si / (kDevelopTile / 2);  // picture tile
        if (atomicOr(p.fb_flags + tile, 1u) == 0) atomicAdd(p.fb_count, 1u);
    }
}

// f32 parameters -> bf16 weights in the tensor cores' B layout, all layers:
// per column offset kx and 16-channel half, two K chunks of N = 3 x cout
// rows (block j of cout rows: kernel row ky = 2 - j) of 8 input channels.
__global__ void k_sg_pack_weights(const float* __restrict__ params, uint16_t* __restrict__ packed) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= kPacked) return;
    int l = 0;
    while (l < kLayers - 1 && i >= packed_off(l + 1)) l++;
    const int cin = cin_of(l), cout = cout_of(l), nb = 3 * cout;
    // k = (((kx * cin/16 + h) * 2 + kc) * nb + n) * 8 + e
    size_t k = i - packed_off(l);
    const int e = int(k % 8);
    k /= 8;
    const int n = int(k % nb);
    k /= nb;
    const int kc = int(k % 2);
    k /= 2;
    const int h = int(k % (cin / 16)), kx = int(k / (cin / 16));
    const int co = n % cout, ky = 2 - n / cout, ci = 16 * h + 8 * kc + e;
    const float wv = params[layer_off(l) + (size_t(co) * cin + ci) * 9 + ky * 3 + kx];
    packed[i] = __bfloat16_as_ushort(__float2bfloat16_rn(wv));
}

// --- training ------------------------------------------------------------------------

struct GatherItem {
    const uint4* in;      // frame input chunks [2][hq][wq], network frame
    const float* base;    // [3][hq][wq], network frame
    const float* target;  // plain develop, white-balanced, planar [3][h][w], picture frame
    int w, h, wq, hq;
    int rr, rc;           // mirrors of the network frame
    int cx, cy;           // crop origin in the network frame, full resolution, even
};

// Window u, v of image k is frame quad (cx/2 - margin + u, cy/2 - margin + v).
__global__ void k_sg_gather(const GatherItem* __restrict__ items, int hw, int ww, int margin, int crop,
                            uint4* __restrict__ in, float* __restrict__ base, float* __restrict__ target,
                            int4* __restrict__ valid) {
    const int k = blockIdx.z;
    const GatherItem it = items[k];
    const int u = blockIdx.x * blockDim.x + threadIdx.x, v = blockIdx.y;
    const int qx0 = it.cx / 2 - margin, qy0 = it.cy / 2 - margin;
    const size_t wplane = size_t(hw) * ww, fplane = size_t(it.wq) * it.hq;
    if (u < ww) {
        const int fx = qx0 + u, fy = qy0 + v;
        const bool inside = fx >= 0 && fy >= 0 && fx < it.wq && fy < it.hq;
        const size_t wi = size_t(k) * 2 * wplane + size_t(v) * ww + u;
        const size_t fi = size_t(fy) * it.wq + fx;
        in[wi] = inside ? it.in[fi] : make_uint4(0, 0, 0, 0);
        in[wi + wplane] = inside ? it.in[fplane + fi] : make_uint4(0, 0, 0, 0);
        for (int c = 0; c < 3; c++)
            base[(size_t(k) * 3 + c) * wplane + size_t(v) * ww + u] = inside ? it.base[c * fplane + fi] : 0.0f;
    }
    // Target crop: rows 2v, 2v+1 of the crop, columns 2u, 2u+1.
    if (u < crop / 2 && v < crop / 2) {
        for (int dy = 0; dy < 2; dy++)
            for (int dx = 0; dx < 2; dx++) {
                const int x = 2 * u + dx, y = 2 * v + dy;
                const int px = it.rc ? it.w - 1 - (it.cx + x) : it.cx + x;
                const int py = it.rr ? it.h - 1 - (it.cy + y) : it.cy + y;
                const size_t fi = size_t(py) * it.w + px;
                for (int c = 0; c < 3; c++)
                    target[((size_t(k) * 3 + c) * crop + y) * crop + x] = it.target[size_t(c) * it.w * it.h + fi];
            }
    }
    if (u == 0 && v == 0 && threadIdx.x == 0) {
        valid[k] = make_int4(max(0, -qx0), max(0, -qy0), min(ww, it.wq - qx0), min(hw, it.hq - qy0));
    }
}

// Loss over the crop (full resolution, at window quad offset `margin`) and
// its gradient with respect to the head. dhead must be zero beforehand.
__global__ void k_sg_loss(const float* __restrict__ head, const float* __restrict__ base,
                          const float* __restrict__ target, int hw, int ww, int margin, int cw, int ch, float scale,
                          float* __restrict__ dhead, double* __restrict__ loss) {
    const int k = blockIdx.z;
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    float local = 0.0f;
    if (x < cw && y < ch) {
        const size_t wplane = size_t(hw) * ww;
        const size_t q = size_t(margin + (y >> 1)) * ww + margin + (x >> 1);
        const int s = (y & 1) * 2 + (x & 1);
        for (int c = 0; c < 3; c++) {
            const size_t hi = (size_t(k) * kHead + c * 4 + s) * wplane + q;
            const float out = head[hi] + base[(size_t(k) * 3 + c) * wplane + q];
            const float d = out - target[((size_t(k) * 3 + c) * ch + y) * cw + x];
            local += d * d;
            dhead[hi] = 2.0f * d * scale;
        }
    }
    for (int o = 16; o > 0; o >>= 1) local += __shfl_xor_sync(0xFFFFFFFFu, local, o);
    __shared__ float part[32];
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = local;
    __syncthreads();
    if (threadIdx.x == 0) {
        float s = 0.0f;
        for (int i = 0; i < int(blockDim.x / 32); i++) s += part[i];
        atomicAdd(loss, double(s));
    }
}

// Gradient of a layer's input through the ReLU that produced it:
// dx[ci] = (x[ci] > 0) * sum_{co, tap} W[co][ci][tap] dy[co][p - tap].
template <int CIN, int COUT>
__global__ void __launch_bounds__(128) k_sg_dx(const float* __restrict__ dy, const float* __restrict__ w,
                                               const uint4* __restrict__ x, int H, int W, float* __restrict__ dx) {
    __shared__ float ws[COUT * 9 * CIN];  // [co][tap][ci]
    for (int i = threadIdx.x; i < COUT * 9 * CIN; i += blockDim.x) {
        const int ci = i % CIN, t = (i / CIN) % 9, co = i / (CIN * 9);
        ws[i] = w[(size_t(co) * CIN + ci) * 9 + t];
    }
    __syncthreads();
    const int img = blockIdx.z;
    const int px = blockIdx.x * 32 + (threadIdx.x & 31), py = blockIdx.y * 4 + (threadIdx.x >> 5);
    if (px >= W || py >= H) return;
    const size_t plane = size_t(H) * W;
    float acc[CIN];
#pragma unroll
    for (int i = 0; i < CIN; i++) acc[i] = 0.0f;
    for (int co = 0; co < COUT; co++) {
        const float* dyc = dy + (size_t(img) * COUT + co) * plane;
#pragma unroll
        for (int t = 0; t < 9; t++) {
            const int oy = py - (t / 3 - 1), ox = px - (t % 3 - 1);
            if (oy < 0 || oy >= H || ox < 0 || ox >= W) continue;
            const float g = __ldg(dyc + size_t(oy) * W + ox);
            const float* wr = ws + (co * 9 + t) * CIN;
#pragma unroll
            for (int ci = 0; ci < CIN; ci++) acc[ci] = fmaf(wr[ci], g, acc[ci]);
        }
    }
    const size_t p = size_t(py) * W + px;
#pragma unroll
    for (int c8 = 0; c8 < CIN / 8; c8++) {
        const uint4 xv = __ldg(x + (size_t(img) * (CIN / 8) + c8) * plane + p);
        const uint32_t words[4] = {xv.x, xv.y, xv.z, xv.w};
#pragma unroll
        for (int e = 0; e < 8; e++) {
            const float xe = (e & 1) ? bf16_hi(words[e >> 1]) : bf16_lo(words[e >> 1]);
            dx[(size_t(img) * CIN + c8 * 8 + e) * plane + p] = xe > 0.0f ? acc[c8 * 8 + e] : 0.0f;
        }
    }
}

// Weight and bias gradients: thread (co group, ci) accumulates CO_T output
// channels x 9 taps over the CTA's tiles of 32 x 8 pixels, then adds them.
template <int CIN, int COUT>
__global__ void __launch_bounds__(128) k_sg_dw(const float* __restrict__ dy, const uint4* __restrict__ x, int H,
                                               int W, int images, float* __restrict__ dw, float* __restrict__ db) {
    constexpr int CO_T = COUT * CIN / 128;
    // Pixel tile 32 x 4; the input with its halo, 6 x 34 per channel, padded
    // to an odd stride so that the 32 channels of a warp fall in 32 banks.
    constexpr int PX = 32, PY = 4, XR = PY + 2, XC = PX + 2, XS = XR * XC + 1;
    __shared__ float xs[CIN * XS];
    __shared__ float ds[COUT * PX * PY];
    const int tid = threadIdx.x;
    const int ci = tid % CIN, cog = tid / CIN;
    float acc[CO_T][9];
    float bacc[CO_T];
#pragma unroll
    for (int a = 0; a < CO_T; a++) {
        bacc[a] = 0.0f;
#pragma unroll
        for (int t = 0; t < 9; t++) acc[a][t] = 0.0f;
    }
    const int tiles_x = (W + PX - 1) / PX, tiles_y = (H + PY - 1) / PY;
    const int ntiles = tiles_x * tiles_y * images;
    const size_t plane = size_t(H) * W;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int img = tile / (tiles_x * tiles_y), rem = tile % (tiles_x * tiles_y);
        const int x0 = (rem % tiles_x) * PX, y0 = (rem / tiles_x) * PY;
        __syncthreads();
        for (int i = tid; i < (CIN / 8) * XR * XC; i += 128) {
            const int c8 = i / (XR * XC), r = (i / XC) % XR, q = i % XC;
            const int gy = y0 - 1 + r, gx = x0 - 1 + q;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (gy >= 0 && gy < H && gx >= 0 && gx < W) v = __ldg(x + (size_t(img) * (CIN / 8) + c8) * plane + size_t(gy) * W + gx);
            const uint32_t words[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
            for (int e = 0; e < 8; e++)
                xs[(c8 * 8 + e) * XS + r * XC + q] = (e & 1) ? bf16_hi(words[e >> 1]) : bf16_lo(words[e >> 1]);
        }
        for (int i = tid; i < COUT * PX * PY; i += 128) {
            const int co = i / (PX * PY), r = (i / PX) % PY, q = i % PX;
            const int gy = y0 + r, gx = x0 + q;
            ds[i] = (gy < H && gx < W) ? __ldg(dy + (size_t(img) * COUT + co) * plane + size_t(gy) * W + gx) : 0.0f;
        }
        __syncthreads();
        for (int r = 0; r < PY; r++)
            for (int q = 0; q < PX; q++) {
                float xv[9];
#pragma unroll
                for (int t = 0; t < 9; t++) xv[t] = xs[ci * XS + (r + t / 3) * XC + q + t % 3];
#pragma unroll
                for (int a = 0; a < CO_T; a++) {
                    const float g = ds[(cog * CO_T + a) * PX * PY + r * PX + q];
                    bacc[a] += g;
#pragma unroll
                    for (int t = 0; t < 9; t++) acc[a][t] = fmaf(xv[t], g, acc[a][t]);
                }
            }
    }
#pragma unroll
    for (int a = 0; a < CO_T; a++) {
        const int co = cog * CO_T + a;
#pragma unroll
        for (int t = 0; t < 9; t++) atomicAdd(dw + (size_t(co) * CIN + ci) * 9 + t, acc[a][t]);
        if (ci == 0) atomicAdd(db + co, bacc[a]);
    }
}

__global__ void k_sg_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                          float* __restrict__ v, size_t n, float lr_t, float b1, float b2, float eps) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr_t * mi / (sqrtf(vi) + eps);
}

// Input chunks from planar f32 (the explicit-image gradient path).
__global__ void k_sg_from_planar(const float* __restrict__ src, int plane, uint4* __restrict__ dst) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= plane) return;
    for (int c8 = 0; c8 < 2; c8++) {
        float f[8];
        for (int e = 0; e < 8; e++) f[e] = src[size_t(c8 * 8 + e) * plane + i];
        dst[size_t(c8) * plane + i] = make_uint4(pack_bf16x2(f[0], f[1]), pack_bf16x2(f[2], f[3]),
                                                 pack_bf16x2(f[4], f[5]), pack_bf16x2(f[6], f[7]));
    }
}

// --- host-side network passes ---------------------------------------------------------

// Buffers of one forward over `images` images of hq x wq pixels.
struct NetBuffers {
    uint4* in = nullptr;      // [images][2][hq][wq]
    uint4* act[6] = {};       // [images][4][hq][wq]
    float* head = nullptr;    // [images][16][hq][wq]
};

// The seven layers; the head writes f32 channels (nb.head), or, given
// `out`, the develop output directly. `fused` runs layers 0-1, 2-3 and 4-5
// as pairs (k_sg_rows2: the first layer of a pair leaves no activations in
// nb.act, so training, which reads them back, runs them one at a time).
cudaError_t forward(const NetBuffers& nb, const uint16_t* packed, const float* params, const int4* valid, int images,
                    int hq, int wq, unsigned* error, cudaStream_t s, const RgbOut* out = nullptr, bool fused = false) {
    const RgbOut none{};
    auto args = [&](int l) {
        ConvArgs a{};
        a.H = hq;
        a.W = wq;
        a.valid = valid;
        a.error = error;
        a.x = l == 0 ? nb.in : nb.act[l - 1];
        a.w = reinterpret_cast<const uint4*>(packed + packed_off(l));
        a.bias = params + layer_off(l) + size_t(cout_of(l)) * cin_of(l) * 9;
        a.y = l < kLayers - 1 ? nb.act[l] : nullptr;
        a.yf = l < kLayers - 1 || out ? nullptr : nb.head;
        return a;
    };
    for (int l = 0; l < kLayers; l++) {
        cudaError_t e;
        if (fused && l < kLayers - 1) {
            e = l == 0 ? conv2_launch<kIn, kHid, kHidden>(args(0), args(1), none, images, s)
                       : conv2_launch<kHid, kHid, kHidden>(args(l), args(l + 1), none, images, s);
            l++;
        } else if (l == 0) {
            e = conv_launch<kIn, kHid, kHidden>(args(l), none, images, s);
        } else if (l < kLayers - 1) {
            e = conv_launch<kHid, kHid, kHidden>(args(l), none, images, s);
        } else if (out) {
            e = conv_launch<kHid, kHead, kHeadRgb>(args(l), *out, images, s);
        } else {
            e = conv_launch<kHid, kHead, kHeadF32>(args(l), none, images, s);
        }
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t pack_weights(const float* params, uint16_t* packed, cudaStream_t s) {
    k_sg_pack_weights<<<unsigned((kPacked + 255) / 256), 256, 0, s>>>(params, packed);
    count_launch();
    return cudaGetLastError();
}

// Backward from dhead: parameter gradients into grad (zeroed here).
cudaError_t backward(const NetBuffers& nb, const float* params, const float* dhead, float* grad, float* d0, float* d1,
                     int images, int hq, int wq, int sms, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(grad, 0, kParams * sizeof(float), s);
    if (e != cudaSuccess) return e;
    const float* dy = dhead;
    float* bufs[2] = {d0, d1};
    const dim3 gdx((wq + 31) / 32, (hq + 3) / 4, images);
    const int gdw = std::max(1, sms * 4);
    for (int l = kLayers - 1; l >= 0; l--) {
        const uint4* x = l == 0 ? nb.in : nb.act[l - 1];
        float* dw = grad + layer_off(l);
        float* db = dw + size_t(cout_of(l)) * cin_of(l) * 9;
        const float* w = params + layer_off(l);
        float* dx = bufs[l & 1];
        if (l == kLayers - 1) {
            k_sg_dw<kHid, kHead><<<gdw, 128, 0, s>>>(dy, x, hq, wq, images, dw, db);
            k_sg_dx<kHid, kHead><<<gdx, 128, 0, s>>>(dy, w, x, hq, wq, dx);
            count_launch(2);
        } else if (l > 0) {
            k_sg_dw<kHid, kHid><<<gdw, 128, 0, s>>>(dy, x, hq, wq, images, dw, db);
            k_sg_dx<kHid, kHid><<<gdx, 128, 0, s>>>(dy, w, x, hq, wq, dx);
            count_launch(2);
        } else {
            k_sg_dw<kIn, kHid><<<gdw, 128, 0, s>>>(dy, x, hq, wq, images, dw, db);
            count_launch();
        }
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        dy = dx;
    }
    return cudaSuccess;
}

}  // namespace sg

// Per-context state of the learned develop: scratch and packed weights.
struct LearnedState {
    DevBuf<uint8_t> scratch;
    DevBuf<uint16_t> packed;
    DevBuf<unsigned> counters;  // [0] fallback tiles, [1] error
    HostBuf<unsigned> hcounters;
};

void learned_state_destroy(LearnedState* s) {
    if (!s) return;
    s->scratch.release();
    s->packed.release();
    s->counters.release();
    s->hcounters.release();
    delete s;
}

}  // namespace prr

// ---------------------------------------------------------------------------
// Trainer.

struct prr_sg_trainer {
    prr_ctx* ctx = nullptr;
    uint32_t batch = 0, crop = 0, margin = 8;
    int sms = 0;
    struct Frame {
        DevBuf<uint4> in;
        DevBuf<float> base;
        DevBuf<float> target;
        int w = 0, h = 0, wq = 0, hq = 0, rr = 0, rc = 0;
    };
    std::vector<Frame*> frames;
    DevBuf<float> params, grad, m, v, minmax;
    DevBuf<uint16_t> packed;
    DevBuf<uint4> win_in;
    DevBuf<uint4> acts;
    DevBuf<float> base, target, head, dhead, d0, d1;
    DevBuf<int4> valid;
    DevBuf<prr::sg::GatherItem> items;
    HostBuf<prr::sg::GatherItem> hitems;
    DevBuf<double> loss;
    DevBuf<unsigned> error;
    HostBuf<double> hloss;
    HostBuf<unsigned> herror;
    HostBuf<float> hminmax;
    uint32_t step = 0;
    float noise_lo = 0.f, noise_hi = 0.f;
    bool have_range = false;
};

using namespace prr;

namespace {

int learned_state(prr_ctx* c, LearnedState** out) {
    if (!c->learned) c->learned = new LearnedState;
    *out = c->learned;
    return PRR_OK;
}

// Pack a decoded frame into the surrogate input and colours; optionally
// the noise channel's range (training) or the fallback tiles of a model
// (fb_flags zeroed beforehand: flags per 32x32 tile, count in fb_count).
int pack_frame(prr_ctx* c, const DevelopDesc& d, uint4* in, float* base, float* minmax, unsigned* fb_flags = nullptr,
               unsigned* fb_count = nullptr, float fb_lo = 0.0f, float fb_hi = 0.0f) {
    sg::PackArgs p{};
    p.codes = d.codes;
    p.stride = d.stride;
    p.w = d.w;
    p.h = d.h;
    p.wq = (d.w + 1) / 2;
    p.hq = (d.h + 1) / 2;
    for (int i = 0; i < 8; i++) {
        p.c0[i] = d.curve_c0[i];
        p.cd[i] = d.curve_delta[i];
    }
    p.rr = d.cfa >> 1;
    p.rc = d.cfa & 1;
    p.black = d.black;
    p.one_over_range = d.one_over_range;
    p.bs = d.green_off;
    p.wb0 = d.wb[0];
    p.wb1 = d.wb[1];
    p.n0 = d.noise[0];
    p.n1 = d.noise[1];
    p.n2 = d.noise[2];
    p.in = in;
    p.base = base;
    p.noise_minmax = minmax;
    p.fb_flags = fb_flags;
    p.fb_count = fb_count;
    p.tiles_x = (d.w + kDevelopTile - 1) / kDevelopTile;
    p.fb_lo = fb_lo;
    p.fb_hi = fb_hi;
    dim3 grid((p.wq + sg::kPackW - 1) / sg::kPackW, (p.hq + sg::kPackH - 1) / sg::kPackH);
    sg::k_sg_pack<<<grid, sg::kPackW * sg::kPackH, 0, c->stream>>>(p);
    count_launch();
    return c->cuda(cudaGetLastError());
}

size_t up256(size_t v) { return (v + 255) & ~size_t(255); }

}  // namespace

extern "C" {

size_t prr_sg_param_count(void) { return sg::kParams; }

int prr_sg_pack(prr_ctx* c, const prr_header* h, const prr_params* params, int stage, const uint16_t* dev_samples,
                float* in16, float* base3) {
    if (!c || !h || !in16 || !base3) return PRR_ERR_INVALID;
    PRR_TRY(c->use_device());
    const int wq = (int(h->width) + 1) / 2, hq = (int(h->height) + 1) / 2;
    const size_t plane = size_t(wq) * hq, n = size_t(h->width) * h->height;
    DevBuf<uint4> in;
    DevBuf<float> base;
    HostBuf<uint4> hin;
    auto cleanup = [&]() {
        in.release();
        base.release();
        hin.release();
    };
    cudaError_t e = in.ensure(2 * plane);
    if (e == cudaSuccess) e = base.ensure(3 * plane);
    if (e == cudaSuccess) e = hin.ensure(2 * plane);
    if (e != cudaSuccess) {
        cleanup();
        return c->cuda(e);
    }
    // The packing reads no output buffer: the input buffer stands in for the
    // interleaved output the descriptor checks (aligned, never written).
    DevelopDesc d{};
    int rc = build_develop_desc(h, params, stage, dev_samples, PRR_INTERLEAVED, reinterpret_cast<float*>(in.p), nullptr,
                                nullptr, 3 * n, &d);
    if (rc == PRR_OK) rc = pack_frame(c, d, in.p, base.p, nullptr);
    if (rc == PRR_OK) {
        e = cudaMemcpyAsync(hin.p, in.p, 2 * plane * sizeof(uint4), cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(base3, base.p, 3 * plane * sizeof(float), cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        rc = c->cuda(e);
    }
    if (rc == PRR_OK) {
        // Chunk k of quad q holds channels 8k .. 8k + 7 as bf16 pairs.
        for (size_t q = 0; q < plane; q++)
            for (int k = 0; k < 2; k++) {
                const uint4 v = hin.p[k * plane + q];
                const uint32_t words[4] = {v.x, v.y, v.z, v.w};
                for (int ch = 0; ch < 8; ch++) {
                    const uint32_t bits = (ch & 1) ? (words[ch >> 1] & 0xFFFF0000u) : (words[ch >> 1] << 16);
                    std::memcpy(in16 + (size_t(8 * k + ch) * plane + q), &bits, 4);
                }
            }
    }
    cleanup();
    return rc;
}

int prr_develop_learned(prr_ctx* c, const prr_header* h, const prr_params* params, int stage,
                        const uint16_t* dev_samples, const prr_sg_model* model, int layout, float* r, float* g,
                        float* b, size_t out_len, uint32_t* fallback_tiles) {
    if (!c || !model || !model->dev_params) return PRR_ERR_INVALID;
    DevelopDesc d{};
    PRR_TRY(build_develop_desc(h, params, stage, dev_samples, layout, r, g, b, out_len, &d));
    PRR_TRY(c->use_device());
    LearnedState* L = nullptr;
    PRR_TRY(learned_state(c, &L));
    const int wq = (d.w + 1) / 2, hq = (d.h + 1) / 2;
    const size_t plane = size_t(wq) * hq;
    const int tiles_x = (d.w + kDevelopTile - 1) / kDevelopTile, tiles_y = (d.h + kDevelopTile - 1) / kDevelopTile;
    const size_t ntiles = size_t(tiles_x) * tiles_y;
    // Scratch: input chunks, colours, two activation buffers, fallback
    // flags per tile (the head writes the output planes itself).
    const size_t o_in = 0, o_base = o_in + up256(plane * 32), o_a0 = o_base + up256(plane * 12),
                 o_a1 = o_a0 + up256(plane * 64), o_mask = o_a1 + up256(plane * 64),
                 total = o_mask + up256(ntiles * sizeof(unsigned));
    PRR_TRY(c->cuda(L->scratch.ensure(total)));
    PRR_TRY(c->cuda(L->packed.ensure(sg::kPacked)));
    PRR_TRY(c->cuda(L->counters.ensure(2)));
    PRR_TRY(c->cuda(L->hcounters.ensure(2)));
    uint8_t* S = L->scratch.p;
    sg::NetBuffers nb;
    nb.in = reinterpret_cast<uint4*>(S + o_in);
    float* base = reinterpret_cast<float*>(S + o_base);
    uint4* a0 = reinterpret_cast<uint4*>(S + o_a0);
    uint4* a1 = reinterpret_cast<uint4*>(S + o_a1);
    // The fused forward writes act[1], act[3], act[5] (each pair's second
    // layer) and reads the one before: they alternate between the buffers.
    for (int l = 0; l < 6; l++) nb.act[l] = ((l >> 1) & 1) ? a1 : a0;
    nb.head = nullptr;
    unsigned* mask = reinterpret_cast<unsigned*>(S + o_mask);
    cudaStream_t s = c->stream;
    PRR_TRY(c->cuda(cudaMemsetAsync(L->counters.p, 0, 2 * sizeof(unsigned), s)));
    PRR_TRY(c->cuda(cudaMemsetAsync(mask, 0, ntiles * sizeof(unsigned), s)));
    // The packing flags the tiles whose noise channel leaves the model's
    // range: the plain develop takes those.
    PRR_TRY(pack_frame(c, d, nb.in, base, nullptr, mask, L->counters.p, model->noise_lo, model->noise_hi));
    PRR_TRY(c->cuda(sg::pack_weights(model->dev_params, L->packed.p, s)));
    sg::RgbOut o{};
    o.base = base;
    o.w = d.w;
    o.h = d.h;
    o.rr = d.cfa >> 1;
    o.rc = d.cfa & 1;
    o.has_matrix = d.has_matrix;
    for (int i = 0; i < 9; i++) o.m[i] = d.m[i];
    o.layout = layout;
    o.r = r;
    o.g = g;
    o.b = b;
    o.fallback = mask;
    o.tiles_x = tiles_x;
    PRR_TRY(c->cuda(sg::forward(nb, L->packed.p, model->dev_params, nullptr, 1, hq, wq, L->counters.p + 1, s, &o, true)));
    PRR_TRY(c->cuda(cudaGetLastError()));
    // The plain develop on the fallback tiles (the others return at once).
    d.tile_mask = mask;
    PRR_TRY(c->cuda(launch_develop(d, s)));
    if (fallback_tiles) {
        PRR_TRY(c->cuda(cudaMemcpyAsync(L->hcounters.p, L->counters.p, 2 * sizeof(unsigned), cudaMemcpyDeviceToHost, s)));
        PRR_TRY(c->cuda(cudaStreamSynchronize(s)));
        *fallback_tiles = L->hcounters.p[0];
        if (L->hcounters.p[1]) return PRR_ERR_TIMEOUT;
    }
    return PRR_OK;
}

int prr_sg_trainer_create(prr_ctx* c, uint32_t batch, uint32_t crop, prr_sg_trainer** out) {
    if (!c || !out || batch == 0 || crop < 32 || (crop & 1)) return PRR_ERR_INVALID;
    PRR_TRY(c->use_device());
    prr_sg_trainer* t = new prr_sg_trainer;
    t->ctx = c;
    t->batch = batch;
    t->crop = crop;
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&t->sms, cudaDevAttrMultiProcessorCount, dev);
    const size_t wq = crop / 2 + 2 * t->margin, plane = wq * wq;
    cudaError_t e = cudaSuccess;
    auto ok = [&](cudaError_t x) { if (e == cudaSuccess) e = x; };
    ok(t->params.ensure(sg::kParams));
    ok(t->grad.ensure(sg::kParams));
    ok(t->m.ensure(sg::kParams));
    ok(t->v.ensure(sg::kParams));
    ok(t->packed.ensure(sg::kPacked));
    ok(t->win_in.ensure(batch * 2 * plane));
    ok(t->acts.ensure(6 * batch * 4 * plane));
    ok(t->base.ensure(batch * 3 * plane));
    ok(t->target.ensure(size_t(batch) * 3 * crop * crop));
    ok(t->head.ensure(batch * 16 * plane));
    ok(t->dhead.ensure(batch * 16 * plane));
    ok(t->d0.ensure(batch * 32 * plane));
    ok(t->d1.ensure(batch * 32 * plane));
    ok(t->valid.ensure(batch));
    ok(t->items.ensure(batch));
    ok(t->hitems.ensure(batch));
    ok(t->loss.ensure(1));
    ok(t->hloss.ensure(1));
    ok(t->error.ensure(1));
    ok(t->herror.ensure(1));
    ok(t->minmax.ensure(2));
    ok(t->hminmax.ensure(2));
    if (e == cudaSuccess) e = cudaMemset(t->m.p, 0, sg::kParams * 4);
    if (e == cudaSuccess) e = cudaMemset(t->v.p, 0, sg::kParams * 4);
    if (e == cudaSuccess) e = cudaMemset(t->params.p, 0, sg::kParams * 4);
    if (e == cudaSuccess) e = cudaMemset(t->error.p, 0, 4);
    if (e != cudaSuccess) {
        prr_sg_trainer_destroy(t);
        return c->cuda(e);
    }
    *out = t;
    return PRR_OK;
}

void prr_sg_trainer_destroy(prr_sg_trainer* t) {
    if (!t) return;
    cudaSetDevice(t->ctx->device);
    cudaStreamSynchronize(t->ctx->stream);
    for (auto* f : t->frames) {
        f->in.release();
        f->base.release();
        f->target.release();
        delete f;
    }
    t->params.release();
    t->grad.release();
    t->m.release();
    t->v.release();
    t->minmax.release();
    t->packed.release();
    t->win_in.release();
    t->acts.release();
    t->base.release();
    t->target.release();
    t->head.release();
    t->dhead.release();
    t->d0.release();
    t->d1.release();
    t->valid.release();
    t->items.release();
    t->hitems.release();
    t->loss.release();
    t->hloss.release();
    t->error.release();
    t->herror.release();
    t->hminmax.release();
    delete t;
}

int prr_sg_trainer_add_frame(prr_sg_trainer* t, const prr_header* h, const prr_params* params,
                             const uint16_t* dev_samples, uint32_t* index) {
    if (!t || !h || !params || !dev_samples) return PRR_ERR_INVALID;
    prr_ctx* c = t->ctx;
    PRR_TRY(c->use_device());
    if (h->width < t->crop || h->height < t->crop) return PRR_ERR_INVALID;
    auto* f = new prr_sg_trainer::Frame;
    f->w = h->width;
    f->h = h->height;
    f->wq = (f->w + 1) / 2;
    f->hq = (f->h + 1) / 2;
    const size_t plane = size_t(f->wq) * f->hq, n = size_t(f->w) * f->h;
    cudaError_t e = f->in.ensure(2 * plane);
    if (e == cudaSuccess) e = f->base.ensure(3 * plane);
    if (e == cudaSuccess) e = f->target.ensure(3 * n);
    if (e != cudaSuccess) {
        delete f;
        return c->cuda(e);
    }
    t->frames.push_back(f);
    // The target: the plain develop, white-balanced stage, planar.
    DevelopDesc d{};
    PRR_TRY(build_develop_desc(h, params, PRR_STAGE_WHITE_BALANCED, dev_samples, PRR_PLANAR, f->target.p,
                               f->target.p + n, f->target.p + 2 * n, n, &d));
    PRR_TRY(c->cuda(launch_develop(d, c->stream)));
    f->rr = d.cfa >> 1;
    f->rc = d.cfa & 1;
    const float init[2] = {__builtin_huge_valf(), 0.0f};
    PRR_TRY(c->cuda(cudaMemcpyAsync(t->minmax.p, init, sizeof(init), cudaMemcpyHostToDevice, c->stream)));
    PRR_TRY(pack_frame(c, d, f->in.p, f->base.p, t->minmax.p));
    PRR_TRY(c->cuda(cudaMemcpyAsync(t->hminmax.p, t->minmax.p, 2 * sizeof(float), cudaMemcpyDeviceToHost, c->stream)));
    PRR_TRY(c->cuda(cudaStreamSynchronize(c->stream)));
    const float lo = t->hminmax.p[0], hi = t->hminmax.p[1];
    t->noise_lo = t->have_range ? std::min(t->noise_lo, lo) : lo;
    t->noise_hi = t->have_range ? std::max(t->noise_hi, hi) : hi;
    t->have_range = true;
    if (index) *index = uint32_t(t->frames.size() - 1);
    return PRR_OK;
}

int prr_sg_trainer_noise_range(prr_sg_trainer* t, float* lo, float* hi) {
    if (!t || !lo || !hi || !t->have_range) return PRR_ERR_INVALID;
    *lo = t->noise_lo;
    *hi = t->noise_hi;
    return PRR_OK;
}

int prr_sg_trainer_set_params(prr_sg_trainer* t, const float* host_params) {
    if (!t || !host_params) return PRR_ERR_INVALID;
    prr_ctx* c = t->ctx;
    PRR_TRY(c->use_device());
    PRR_TRY(c->cuda(cudaMemcpy(t->params.p, host_params, sg::kParams * 4, cudaMemcpyHostToDevice)));
    PRR_TRY(c->cuda(cudaMemset(t->m.p, 0, sg::kParams * 4)));
    PRR_TRY(c->cuda(cudaMemset(t->v.p, 0, sg::kParams * 4)));
    t->step = 0;
    return PRR_OK;
}

int prr_sg_trainer_get_params(prr_sg_trainer* t, float* host_params) {
    if (!t || !host_params) return PRR_ERR_INVALID;
    prr_ctx* c = t->ctx;
    PRR_TRY(c->use_device());
    PRR_TRY(c->cuda(cudaStreamSynchronize(c->stream)));
    return c->cuda(cudaMemcpy(host_params, t->params.p, sg::kParams * 4, cudaMemcpyDeviceToHost));
}

const float* prr_sg_trainer_device_params(prr_sg_trainer* t) { return t ? t->params.p : nullptr; }

int prr_sg_trainer_step(prr_sg_trainer* t, const uint32_t* crops, float lr, float* loss_out) {
    if (!t || !crops) return PRR_ERR_INVALID;
    prr_ctx* c = t->ctx;
    PRR_TRY(c->use_device());
    cudaStream_t s = c->stream;
    const int B = int(t->batch), crop = int(t->crop), M = int(t->margin);
    const int ww = crop / 2 + 2 * M, hw = ww;
    const size_t plane = size_t(ww) * hw;
    // The host items array is read by the copy below: wait for the last one.
    PRR_TRY(c->cuda(cudaStreamSynchronize(s)));
    for (int k = 0; k < B; k++) {
        const uint32_t fi = crops[3 * k], cx = crops[3 * k + 1], cy = crops[3 * k + 2];
        if (fi >= t->frames.size()) return PRR_ERR_INVALID;
        const auto* f = t->frames[fi];
        if ((cx & 1) || (cy & 1) || cx + uint32_t(crop) > uint32_t(f->w) || cy + uint32_t(crop) > uint32_t(f->h))
            return PRR_ERR_INVALID;
        sg::GatherItem& it = t->hitems.p[k];
        it.in = f->in.p;
        it.base = f->base.p;
        it.target = f->target.p;
        it.w = f->w;
        it.h = f->h;
        it.wq = f->wq;
        it.hq = f->hq;
        it.rr = f->rr;
        it.rc = f->rc;
        it.cx = int(cx);
        it.cy = int(cy);
    }
    PRR_TRY(c->cuda(cudaMemcpyAsync(t->items.p, t->hitems.p, B * sizeof(sg::GatherItem), cudaMemcpyHostToDevice, s)));
    sg::k_sg_gather<<<dim3((ww + 127) / 128, hw, B), 128, 0, s>>>(t->items.p, hw, ww, M, crop, t->win_in.p, t->base.p,
                                                                   t->target.p, t->valid.p);
    count_launch();
    sg::NetBuffers nb;
    nb.in = t->win_in.p;
    for (int l = 0; l < 6; l++) nb.act[l] = t->acts.p + size_t(l) * B * 4 * plane;
    nb.head = t->head.p;
    PRR_TRY(c->cuda(sg::pack_weights(t->params.p, t->packed.p, s)));
    PRR_TRY(c->cuda(sg::forward(nb, t->packed.p, t->params.p, t->valid.p, B, hw, ww, t->error.p, s)));
    PRR_TRY(c->cuda(cudaMemsetAsync(t->dhead.p, 0, size_t(B) * 16 * plane * 4, s)));
    PRR_TRY(c->cuda(cudaMemsetAsync(t->loss.p, 0, sizeof(double), s)));
    const float scale = float(1.0 / (3.0 * B * double(crop) * crop));
    sg::k_sg_loss<<<dim3((crop + 127) / 128, crop, B), 128, 0, s>>>(t->head.p, t->base.p, t->target.p, hw, ww, M, crop,
                                                                     crop, scale, t->dhead.p, t->loss.p);
    count_launch();
    PRR_TRY(c->cuda(sg::backward(nb, t->params.p, t->dhead.p, t->grad.p, t->d0.p, t->d1.p, B, hw, ww, t->sms, s)));
    t->step++;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const double bc1 = 1.0 - std::pow(double(b1), double(t->step)), bc2 = 1.0 - std::pow(double(b2), double(t->step));
    const float lr_t = float(lr * std::sqrt(bc2) / bc1);
    sg::k_sg_adam<<<unsigned((sg::kParams + 255) / 256), 256, 0, s>>>(t->params.p, t->grad.p, t->m.p, t->v.p, sg::kParams,
                                                                      lr_t, b1, b2, eps);
    count_launch();
    PRR_TRY(c->cuda(cudaGetLastError()));
    if (loss_out) {
        PRR_TRY(c->cuda(cudaMemcpyAsync(t->hloss.p, t->loss.p, sizeof(double), cudaMemcpyDeviceToHost, s)));
        PRR_TRY(c->cuda(cudaMemcpyAsync(t->herror.p, t->error.p, sizeof(unsigned), cudaMemcpyDeviceToHost, s)));
        PRR_TRY(c->cuda(cudaStreamSynchronize(s)));
        *loss_out = float(t->hloss.p[0] / (3.0 * B * double(crop) * crop));
        if (t->herror.p[0]) return PRR_ERR_TIMEOUT;
    }
    return PRR_OK;
}

int prr_sg_gradients(prr_ctx* c, const float* in16, const float* base3, const float* target3, uint32_t hq, uint32_t wq,
                     const float* params, float* head_out, float* dparams, double* loss_out) {
    if (!c || !in16 || !base3 || !target3 || !params || hq == 0 || wq == 0) return PRR_ERR_INVALID;
    PRR_TRY(c->use_device());
    cudaStream_t s = c->stream;
    const size_t plane = size_t(hq) * wq;
    const int w = int(2 * wq), h = int(2 * hq);
    DevBuf<float> fin, fbase, ftarget, fparams, fhead, fdhead, fgrad, d0, d1, fplanar;
    DevBuf<uint4> in, acts;
    DevBuf<uint16_t> packed;
    DevBuf<double> loss;
    DevBuf<unsigned> err;
    auto cleanup = [&]() {
        fin.release(); fbase.release(); ftarget.release(); fparams.release(); fhead.release(); fdhead.release();
        fgrad.release(); d0.release(); d1.release(); fplanar.release(); in.release(); acts.release();
        packed.release(); loss.release(); err.release();
    };
    cudaError_t e = cudaSuccess;
    auto ok = [&](cudaError_t x) { if (e == cudaSuccess) e = x; };
    ok(fplanar.ensure(16 * plane));
    ok(fbase.ensure(3 * plane));
    ok(ftarget.ensure(3 * size_t(w) * h));
    ok(fparams.ensure(sg::kParams));
    ok(fhead.ensure(16 * plane));
    ok(fdhead.ensure(16 * plane));
    ok(fgrad.ensure(sg::kParams));
    ok(d0.ensure(32 * plane));
    ok(d1.ensure(32 * plane));
    ok(in.ensure(2 * plane));
    ok(acts.ensure(6 * 4 * plane));
    ok(packed.ensure(sg::kPacked));
    ok(loss.ensure(1));
    ok(err.ensure(1));
    ok(cudaMemcpyAsync(fplanar.p, in16, 16 * plane * 4, cudaMemcpyHostToDevice, s));
    ok(cudaMemcpyAsync(fbase.p, base3, 3 * plane * 4, cudaMemcpyHostToDevice, s));
    ok(cudaMemcpyAsync(ftarget.p, target3, 3 * size_t(w) * h * 4, cudaMemcpyHostToDevice, s));
    ok(cudaMemcpyAsync(fparams.p, params, sg::kParams * 4, cudaMemcpyHostToDevice, s));
    ok(cudaMemsetAsync(fdhead.p, 0, 16 * plane * 4, s));
    ok(cudaMemsetAsync(loss.p, 0, 8, s));
    ok(cudaMemsetAsync(err.p, 0, 4, s));
    if (e != cudaSuccess) {
        cleanup();
        return c->cuda(e);
    }
    sg::k_sg_from_planar<<<unsigned((plane + 127) / 128), 128, 0, s>>>(fplanar.p, int(plane), in.p);
    count_launch();
    sg::NetBuffers nb;
    nb.in = in.p;
    for (int l = 0; l < 6; l++) nb.act[l] = acts.p + size_t(l) * 4 * plane;
    nb.head = fhead.p;
    ok(sg::pack_weights(fparams.p, packed.p, s));
    ok(sg::forward(nb, packed.p, fparams.p, nullptr, 1, int(hq), int(wq), err.p, s));
    const float scale = float(1.0 / (3.0 * double(w) * h));
    sg::k_sg_loss<<<dim3((w + 127) / 128, h, 1), 128, 0, s>>>(fhead.p, fbase.p, ftarget.p, int(hq), int(wq), 0, w, h,
                                                               scale, fdhead.p, loss.p);
    count_launch();
    int sms = 148;
    ok(sg::backward(nb, fparams.p, fdhead.p, fgrad.p, d0.p, d1.p, 1, int(hq), int(wq), sms, s));
    double hl = 0.0;
    unsigned he = 0;
    if (head_out) ok(cudaMemcpyAsync(head_out, fhead.p, 16 * plane * 4, cudaMemcpyDeviceToHost, s));
    if (dparams) ok(cudaMemcpyAsync(dparams, fgrad.p, sg::kParams * 4, cudaMemcpyDeviceToHost, s));
    ok(cudaMemcpyAsync(&hl, loss.p, 8, cudaMemcpyDeviceToHost, s));
    ok(cudaMemcpyAsync(&he, err.p, 4, cudaMemcpyDeviceToHost, s));
    ok(cudaStreamSynchronize(s));
    cleanup();
    if (e != cudaSuccess) return c->cuda(e);
    if (loss_out) *loss_out = hl / (3.0 * double(w) * h);
    return he ? PRR_ERR_TIMEOUT : PRR_OK;
}

}  // extern "C"

namespace prr {

// A 2-D tensor map of 16-bit elements: `width` x `height`, rows `row_bytes`
// apart (a multiple of 16), boxes of box_w x box_h, no swizzle.
cudaError_t encode_u16_map_2d(CUtensorMap* map, const void* base, uint64_t width, uint64_t height,
                              uint64_t row_bytes, uint32_t box_w, uint32_t box_h) {
    const sg::EncodeTiledFn fn = sg::encode_tiled();
    if (!fn) return cudaErrorUnknown;
    const cuuint64_t dims[2] = {width, height};
    const cuuint64_t strides[1] = {row_bytes};
    const cuuint32_t box[2] = {box_w, box_h};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT16, 2, const_cast<void*>(base), dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

}  // namespace prr
