// device_common.cuh -- device building blocks of the decode path: codebook
// tables, the 64-bit window bit reader, the codeword decoder, component
// entropy decoding and the inverse transforms.
//
// Everything here reproduces the crate's integer and f32 arithmetic bit for
// bit (src/bits.rs, src/codebook.rs, src/coefficients.rs, src/idct.rs).
// Float operations are written with the _rn intrinsics so that no multiply
// is ever fused with an addition, whatever the compiler flags.
#pragma once

#include <cstdint>

namespace prr {

// ---------------------------------------------------------------------------
// Codebook tables (src/codebook.rs:25-110), staged into shared memory by each
// CTA: lookups are indexed by per-thread symbols, which constant memory would
// serialize.
constexpr uint16_t FIRST_DC = 0x2BC;
constexpr uint16_t DC_RESET = 0x064;
constexpr uint16_t AC_INITIAL = 0x031;
constexpr uint16_t RN_INITIAL = 0x000;
constexpr uint16_t LN_INITIAL = 0x042;

struct CodeTables {
    uint16_t ac[96];
    uint16_t rn[28];
    uint16_t ln[16];
    uint16_t dc[16];
    uint8_t scan[64];
    uint8_t scan4[16];
    uint8_t scan2[4];
    uint8_t pad[12];
};

__constant__ CodeTables c_tables = {
    {0x000, 0x211, 0x111, 0x111, 0x222, 0x222, 0x222, 0x122, 0x122, 0x122, 0x233, 0x233,
     0x233, 0x233, 0x233, 0x233, 0x233, 0x233, 0x133, 0x133, 0x244, 0x244, 0x244, 0x244,
     0x244, 0x244, 0x244, 0x244, 0x244, 0x244, 0x244, 0x244, 0x244, 0x244, 0x244, 0x244,
     0x244, 0x244, 0x244, 0x244, 0x244, 0x244, 0x355, 0x355, 0x355, 0x355, 0x355, 0x355,
     0x355, 0x355, 0x355, 0x355, 0x355, 0x355, 0x355, 0x355, 0x355, 0x355, 0x355, 0x355,
     0x355, 0x355, 0x355, 0x355, 0x355, 0x355, 0x355, 0x355, 0x355, 0x355, 0x355, 0x355,
     0x355, 0x355, 0x355, 0x355, 0x355, 0x355, 0x355, 0x355, 0x355, 0x355, 0x355, 0x355,
     0x355, 0x355, 0x355, 0x355, 0x355, 0x355, 0x355, 0x355, 0x355, 0x355, 0x166, 0x166},
    {0x200, 0x100, 0x000, 0x000, 0x211, 0x211, 0x111, 0x111, 0x011, 0x011, 0x021, 0x021, 0x222, 0x022,
     0x022, 0x022, 0x022, 0x022, 0x022, 0x022, 0x022, 0x022, 0x022, 0x022, 0x022, 0x032, 0x032, 0x044},
    {0x100, 0x111, 0x222, 0x222, 0x122, 0x122, 0x433, 0x433, 0x233, 0x233, 0x233, 0x233, 0x233,
     0x233, 0x033, 0x033},
    {0x010, 0x021, 0x032, 0x033, 0x033, 0x033, 0x044, 0x044, 0x044, 0x044, 0x044, 0x044, 0x076,
     0x076, 0x076, 0x076},
    {0,  8,  1,  9,  16, 24, 17, 25, 2,  10, 3,  11, 18, 26, 19, 27, 32, 40, 33, 34, 41, 48,
     56, 49, 42, 35, 43, 50, 57, 58, 51, 59, 4,  12, 5,  6,  13, 20, 28, 21, 14, 7,  15, 22,
     29, 36, 44, 37, 30, 23, 31, 38, 45, 52, 60, 53, 46, 39, 47, 54, 61, 62, 55, 63},
    {0, 4, 1, 5, 8, 12, 9, 13, 2, 6, 3, 7, 10, 14, 11, 15},
    {0, 2, 1, 3},
    {0},
};

// Copy the tables to shared memory (all threads of the CTA participate).
__device__ __forceinline__ void load_tables(CodeTables* s) {
    const uint32_t* src = reinterpret_cast<const uint32_t*>(&c_tables);
    uint32_t* dst = reinterpret_cast<uint32_t*>(s);
    for (uint32_t i = threadIdx.x; i < sizeof(CodeTables) / 4; i += blockDim.x) dst[i] = src[i];
}

// ---------------------------------------------------------------------------
// Packet access. The packet is a 4-byte aligned device buffer read as 32-bit
// words; `be_bytes` reads n (0..4) bytes at byte offset p as the top bytes of
// a big-endian word and touches only the aligned words holding those bytes.
__device__ __forceinline__ uint32_t bswap32(uint32_t w) { return __byte_perm(w, 0, 0x0123); }

__device__ __forceinline__ uint32_t be_bytes(const uint32_t* __restrict__ words, uint32_t p, uint32_t n) {
    if (n == 0) return 0;
    const uint32_t sh = (p & 3) * 8;
    uint32_t v = bswap32(__ldg(words + (p >> 2))) << sh;
    if ((p & 3) + n > 4) v |= bswap32(__ldg(words + (p >> 2) + 1)) >> (32 - sh);
    return v & (0xFFFFFFFFu << (32 - 8 * n));
}

__device__ __forceinline__ uint32_t byte_at(const uint32_t* __restrict__ words, uint32_t p) {
    return (__ldg(words + (p >> 2)) >> ((p & 3) * 8)) & 0xFF;
}

__device__ __forceinline__ uint32_t be16_at(const uint32_t* __restrict__ words, uint32_t p) {
    return (byte_at(words, p) << 8) | byte_at(words, p + 1);
}

// Word sources of the bit reader: the packet in global memory, or a copy of
// a span of it in shared memory (words `base` onwards), indexed by the
// packet's word index either way.
struct GlobalWords {
    const uint32_t* w;
    __device__ __forceinline__ uint32_t operator()(uint32_t i) const { return __ldg(w + i); }
};
struct SharedWords {
    const uint32_t* w;
    uint32_t base;
    __device__ __forceinline__ uint32_t operator()(uint32_t i) const { return w[i - base]; }
};

template <class Src>
__device__ __forceinline__ uint32_t be_bytes_src(const Src& src, uint32_t p, uint32_t n) {
    if (n == 0) return 0;
    const uint32_t sh = (p & 3) * 8;
    uint32_t v = bswap32(src(p >> 2)) << sh;
    if ((p & 3) + n > 4) v |= bswap32(src((p >> 2) + 1)) >> (32 - sh);
    return v & (0xFFFFFFFFu << (32 - 8 * n));
}

// ---------------------------------------------------------------------------
// Bit reader, src/bits.rs:17-112: a 64-bit window whose top 32 bits are the
// view, a signed count of valid bits below it, one aligned big-endian word
// per refill, zero fill past the end. The next refill word is fetched one
// refill ahead and touched only by the next refill.
template <class Src>
struct Reader {
    Src src;
    uint32_t words_end;  // whole words may be loaded while pos < words_end
    uint32_t end;        // one past the stream's last byte (packet offsets)
    uint32_t nxt;        // the value the next refill returns
    uint32_t nxt_pos;    // the position after that refill
    uint64_t window;
    int32_t extra;

    __device__ __forceinline__ void peek(uint32_t p) {
        if (p < words_end) {
            nxt = bswap32(src(p >> 2));
            nxt_pos = p + 4;
        } else {
            nxt = be_bytes_src(src, p, end - p);
            nxt_pos = end;
        }
    }

    // BitReader::new (src/bits.rs:44-76) for `len` bytes at packet offset
    // `off`; the stream's alignment is off & 3 (the packet counts as aligned,
    // src/decoder.rs:288-291).
    __device__ __forceinline__ void init(const Src& s, uint32_t off, uint32_t len) {
        src = s;
        end = off + len;
        uint32_t remaining = len;
        uint32_t pos;
        uint32_t first;
        if (remaining < 4) {
            first = be_bytes_src(src, off, remaining);
            pos = off + remaining;
            remaining = 0;
        } else {
            first = be_bytes_src(src, off, 4);
            pos = off + 4;
            remaining -= 4;
        }
        uint32_t low = 0;
        extra = 0;
        const uint32_t to_boundary = (4 - (pos & 3)) & 3;
        if (to_boundary != 0 && to_boundary <= remaining) {
            low = be_bytes_src(src, pos, to_boundary);
            pos += to_boundary;
            remaining -= to_boundary;
            extra = int32_t(8 * to_boundary);
        }
        words_end = pos + 4 * (remaining / 4);
        window = (uint64_t(first) << 32) | uint64_t(low);
        peek(pos);
    }

    __device__ __forceinline__ uint32_t top() const { return uint32_t(window >> 32); }

    // BitReader::consume (src/bits.rs:97-105): drop n bits, refilling at
    // most once.
    __device__ __forceinline__ void consume(uint32_t n) {
        window <<= (n & 63);
        extra = int32_t(uint32_t(extra) - n);
        if (extra < 0) {
            const uint32_t shift = uint32_t(-int32_t(int8_t(extra))) & 63;
            window |= uint64_t(nxt) << shift;
            extra += 32;
            peek(nxt_pos);
        }
    }
};

// codeword, src/bits.rs:116-134, for a view p != 0: value and length. The
// Rice and exp-Golomb results are both computed and one is selected, so
// lanes decoding different kinds of codeword do not diverge. (The crate's
// separate branch for a set top bit is the Rice case with no leading zero.)
__device__ __forceinline__ uint32_t codeword(uint32_t p, uint32_t cb, uint32_t& len) {
    const uint32_t r = cb & 15;
    const uint32_t s = cb >> 8;
    const uint32_t e = (cb >> 4) & 15;
    const uint32_t lz = __clz(p);
    const uint32_t rice_len = r + 1 + lz;
    const uint32_t rice_val = (lz << r) + (((p << ((lz + 1) & 31)) >> 1) >> ((31u - r) & 31));
    const uint32_t eg_len = 2 * lz - s + e;
    const uint32_t eg_val = ((s + 1) << r) + (p >> ((32u - eg_len) & 31)) - (1u << e);
    const bool rice = lz <= s;
    len = rice ? rice_len : eg_len;
    return rice ? rice_val : eg_val;
}

// decode_component_reduced, src/coefficients.rs:37-146, as a state machine
// that decodes one symbol per iteration: the DC fold, the DC deltas, the
// non-zero run length, the levels of a run, the zero run and the level after
// it. Every lane of a warp runs the same codeword and consume for its own
// stream, whatever state its stream is in; only the short per-state updates
// differ. The destination must hold zeros; `store(index, value)` receives
// each coefficient written, index = block * (1 << log2_coefs) + position
// within the block's corner. A wrapped zero run may revisit an index (the
// later store wins, as on the host) and sets `revisited`. Returns false if
// the iteration bound was hit, which no stream of `len` bytes reaches: every
// symbol shifts the window or moves the reader a word on.
template <class Src, class Store>
__device__ __forceinline__ bool decode_component(const Src& src, uint32_t off, uint32_t len,
                                                 uint32_t log2_blocks, uint32_t log2_coefs,
                                                 const CodeTables& T, Store store, bool& revisited) {
    enum : uint32_t { FIRST, DC, RUN_LENGTH, LEVELS, ZEROS, LEVEL, };
    const uint8_t* scan = log2_coefs == 6 ? T.scan : (log2_coefs == 4 ? T.scan4 : T.scan2);
    const uint32_t blocks = 1u << log2_blocks;
    const uint32_t codes = blocks << log2_coefs;
    const uint32_t block_mask = blocks - 1;
    Reader<Src> r;
    r.init(src, off, len);
    uint32_t state = FIRST, cb = FIRST_DC;
    int32_t dc = 0;
    uint32_t sign = 0, block = 1;
    uint32_t ac_cb = AC_INITIAL, rn_cb = RN_INITIAL, ln_cb = LN_INITIAL;
    uint32_t n = blocks, run = 0;
    uint32_t budget = 64u * (8u * len + 64u) + 4u * codes;
    for (;;) {
        const uint32_t top = r.top();
        if (top == 0) return true;  // end of component: the rest stays zero
        if (budget-- == 0) return false;
        uint32_t l;
        const uint32_t v = codeword(top, cb, l);
        const bool is_level = state == LEVELS || state == LEVEL;
        // A level's sign is the bit after its codeword (src/coefficients.rs:90-104).
        const bool negative = int32_t(top << (l & 31)) < 0;
        r.consume(l + (is_level ? 1u : 0u));
        if (is_level) {
            const uint16_t mag = uint16_t(uint16_t(v) + 1);
            const int16_t value = int16_t(negative ? uint16_t(0u - mag) : mag);
            ac_cb = T.ac[min(v, 94u)];
            store(uint32_t(scan[n >> log2_blocks]) + ((n & block_mask) << log2_coefs), value);
            n += 1;
            if (state == LEVEL) {
                ln_cb = T.ln[min(v, 14u)];
                if (n >= codes) return true;
                state = RUN_LENGTH;
                cb = ln_cb;
            } else {
                if (n == codes) return true;
                run -= 1;
                state = run == 0 ? ZEROS : LEVELS;
                cb = run == 0 ? rn_cb : ac_cb;
            }
        } else if (state == RUN_LENGTH) {
            run = v;
            state = run > 0 ? LEVELS : ZEROS;
            cb = run > 0 ? ac_cb : rn_cb;
        } else if (state == ZEROS) {
            rn_cb = T.rn[min(v, 27u)];
            const uint32_t before = n;
            n = n + 1 + v;  // a zero run is zeros + 1 long; wraps like the crate's u32
            if (n < before) revisited = true;
            if (n >= codes) return true;
            state = LEVEL;
            cb = ac_cb;
        } else if (state == DC) {
            sign ^= v & 1;
            const uint32_t magnitude = ((v & 1) + v) >> 1;
            const int32_t delta = int32_t(((0u - sign) ^ magnitude) + sign);
            sign = delta < 0 ? 1u : 0u;
            dc = int32_t(uint32_t(dc) + uint32_t(delta));
            store(block << log2_coefs, int16_t(dc));
            block += 1;
            const uint32_t next_dc = T.dc[min(magnitude, 12u)];
            state = block == blocks ? RUN_LENGTH : DC;
            cb = block == blocks ? ln_cb : next_dc;
        } else {  // FIRST: the sign-folded first DC
            const uint32_t odd = v & 1;
            dc = int32_t((((odd + v) >> 1) ^ (0u - odd)) + odd);
            store(0u, int16_t(dc));
            state = blocks > 1 ? DC : RUN_LENGTH;
            cb = blocks > 1 ? uint32_t(DC_RESET) : ln_cb;
        }
    }
}

// dequantize, src/idct.rs:41-43: 32-bit product saturated to 16 bits.
__device__ __forceinline__ int16_t dequantize(int32_t coef, int32_t q) {
    return int16_t(min(max(coef * q, -32768), 32767));
}

// ---------------------------------------------------------------------------
// Apple-compatible transform, src/idct.rs:51-174.
__constant__ int32_t c_row_tables[4][4][8] = {
    {{4096, 5352, 4096, 2217, 4096, -2217, 4096, -5352},
     {4096, 2217, -4096, -5352, -4096, 5352, 4096, -2217},
     {5681, 4816, 4816, -1130, 3218, -5681, 1130, -3218},
     {3218, 1130, -5681, -3218, 1130, 4816, 4816, -5681}},
    {{5681, 7423, 5681, 3075, 5681, -3075, 5681, -7423},
     {5681, 3075, -5681, -7423, -5681, 7423, 5681, -3075},
     {7880, 6681, 6681, -1567, 4464, -7880, 1567, -4464},
     {4464, 1567, -7880, -4464, 1567, 6681, 6681, -7880}},
    {{5352, 6992, 5352, 2896, 5352, -2896, 5352, -6992},
     {5352, 2896, -5352, -6992, -5352, 6992, 5352, -2896},
     {7423, 6293, 6293, -1477, 4205, -7423, 1477, -4205},
     {4205, 1477, -7423, -4205, 1477, 6293, 6293, -7423}},
    {{4816, 6293, 4816, 2607, 4816, -2607, 4816, -6293},
     {4816, 2607, -4816, -6293, -4816, 6293, 4816, -2607},
     {6681, 5663, 5663, -1329, 3784, -6681, 1329, -3784},
     {3784, 1329, -6681, -3784, 1329, 5663, 5663, -6681}},
};
__host__ __device__ constexpr int row_set(int row) {
    return (row & 3) == 0 ? 0 : (row < 4 ? row : 8 - row);  // {0,1,2,3,0,3,2,1}
}

__device__ __forceinline__ float f32_bits(uint32_t u) { return __uint_as_float(u); }
#define PRR_SCALE f32_bits(0x39800000u)  /* 2^-12 */
#define PRR_SCALE4 f32_bits(0x39000000u) /* 2^-13 */
#define PRR_BIAS f32_bits(0x47000080u)   /* 32768.5 */
#define PRR_TAN1 f32_bits(0x3e4bafafu)
#define PRR_TAN2 f32_bits(0x3ed413cdu)
#define PRR_TAN3 f32_bits(0x3f2b0dc1u)
#define PRR_COS4 f32_bits(0x3f3504f3u)

// Row pass of row `row` (dequantized int16 inputs): eight f32 outputs
// (int32 result rounded to f32, times 2^-12). The row's table set is uniform
// across a warp when the warp works on one row index.
__device__ __forceinline__ void apple_row(const int16_t* x16, int row, float* out) {
    const int32_t(*t)[8] = c_row_tables[row_set(row)];
    int32_t x[8];
#pragma unroll
    for (int i = 0; i < 8; i++) x[i] = x16[i];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const int32_t even = x[0] * t[0][2 * k] + x[2] * t[0][2 * k + 1] + x[4] * t[1][2 * k] +
                             x[6] * t[1][2 * k + 1];
        const int32_t odd = x[1] * t[2][2 * k] + x[3] * t[2][2 * k + 1] + x[5] * t[3][2 * k] +
                            x[7] * t[3][2 * k + 1];
        out[k] = __fmul_rn(__int2float_rn(even + odd), PRR_SCALE);
        out[7 - k] = __fmul_rn(__int2float_rn(even - odd), PRR_SCALE);
    }
}

// trunc_to_i32 + output_code, src/idct.rs:109-123.
__device__ __forceinline__ uint16_t output_code(float v) {
    int32_t t = (v >= -2147483648.0f && v < 2147483648.0f) ? __float2int_rz(v) : INT32_MIN;
    int32_t centred = int32_t(uint32_t(t) - 32768u);
    centred = min(max(centred, -32768), 32767);
    return uint16_t(uint16_t(int16_t(centred)) ^ 0x8000u);
}

// Column pass of one column r[0..7] (src/idct.rs:136-172), in the host's
// order, every operation rounded on its own.
__device__ __forceinline__ void apple_col(const float* r, uint16_t* out) {
    const float p = __fadd_rn(r[0], PRR_BIAS);
    const float ea = __fadd_rn(p, r[4]);
    const float eb = __fsub_rn(p, r[4]);
    const float f = __fadd_rn(__fmul_rn(r[6], PRR_TAN2), r[2]);
    const float g = __fsub_rn(__fmul_rn(r[2], PRR_TAN2), r[6]);
    const float e0 = __fadd_rn(ea, f), e3 = __fsub_rn(ea, f);
    const float e1 = __fadd_rn(eb, g), e2 = __fsub_rn(eb, g);
    const float a = __fadd_rn(__fmul_rn(r[7], PRR_TAN1), r[1]);
    const float b = __fsub_rn(__fmul_rn(r[1], PRR_TAN1), r[7]);
    const float c = __fadd_rn(__fmul_rn(r[5], PRR_TAN3), r[3]);
    const float d = __fsub_rn(r[5], __fmul_rn(r[3], PRR_TAN3));
    const float o0 = __fadd_rn(a, c), t = __fsub_rn(a, c);
    const float o3 = __fadd_rn(b, d), u = __fsub_rn(b, d);
    const float o1 = __fmul_rn(__fadd_rn(t, u), PRR_COS4);
    const float o2 = __fmul_rn(__fsub_rn(t, u), PRR_COS4);
    out[0] = output_code(__fadd_rn(e0, o0));
    out[1] = output_code(__fadd_rn(e1, o1));
    out[2] = output_code(__fadd_rn(e2, o2));
    out[3] = output_code(__fadd_rn(e3, o3));
    out[4] = output_code(__fsub_rn(e3, o3));
    out[5] = output_code(__fsub_rn(e2, o2));
    out[6] = output_code(__fsub_rn(e1, o1));
    out[7] = output_code(__fsub_rn(e0, o0));
}

// 4x4 transform, src/idct.rs:176-226.
__device__ __forceinline__ void apple_row4(const int16_t* x16, int row, float* out) {
    const int32_t k = (row & 1) ? 10703 : 8192;
    const int32_t t0 = (row & 1) ? 13985 : 10703, t1 = (row & 1) ? 5793 : 4433;
    const int32_t t2 = t1, t3 = -t0;
    const int32_t x0 = x16[0], x1 = x16[1], x2 = x16[2], x3 = x16[3];
    const int32_t e0 = k * x0 + k * x2, e1 = k * x0 - k * x2;
    const int32_t o0 = t0 * x1 + t1 * x3, o1 = t2 * x1 + t3 * x3;
    out[0] = __fmul_rn(__int2float_rn(e0 + o0), PRR_SCALE4);
    out[1] = __fmul_rn(__int2float_rn(e1 + o1), PRR_SCALE4);
    out[2] = __fmul_rn(__int2float_rn(e1 - o1), PRR_SCALE4);
    out[3] = __fmul_rn(__int2float_rn(e0 - o0), PRR_SCALE4);
}
__device__ __forceinline__ void apple_col4(const float* r, uint16_t* out) {
    const float r0 = __fadd_rn(r[0], PRR_BIAS);
    const float e0 = __fadd_rn(r[2], r0), e1 = __fsub_rn(r0, r[2]);
    const float f = __fadd_rn(__fmul_rn(r[3], PRR_TAN2), r[1]);
    const float g = __fsub_rn(__fmul_rn(r[1], PRR_TAN2), r[3]);
    out[0] = output_code(__fadd_rn(f, e0));
    out[1] = output_code(__fadd_rn(g, e1));
    out[2] = output_code(__fsub_rn(e1, g));
    out[3] = output_code(__fsub_rn(e0, f));
}

// saturate_code + 2x2 transform, src/idct.rs:189-247 (inputs dequantized).
__device__ __forceinline__ uint16_t saturate_code(int32_t v) {
    return uint16_t(uint16_t(int16_t(min(max(v, -32768), 32767))) ^ 0x8000u);
}
__device__ __forceinline__ void apple_2x2(int32_t d0, int32_t d1, int32_t d2, int32_t d3, uint16_t* out) {
    const int32_t ts = d0 + d1, td = d0 - d1, bs = d2 + d3, bd = d2 - d3;
    out[0] = saturate_code(ts + bs);
    out[1] = saturate_code(td + bd);
    out[2] = saturate_code(ts - bs);
    out[3] = saturate_code(td - bd);
}

// ---------------------------------------------------------------------------
// FFmpeg simple IDCT, src/idct.rs:252-351 (wrapping 32-bit arithmetic).
__device__ __forceinline__ int32_t wmul(int32_t a, int32_t b) { return int32_t(uint32_t(a) * uint32_t(b)); }
__device__ __forceinline__ int32_t wadd(int32_t a, int32_t b) { return int32_t(uint32_t(a) + uint32_t(b)); }
__device__ __forceinline__ int32_t wsub(int32_t a, int32_t b) { return int32_t(uint32_t(a) - uint32_t(b)); }

__device__ __forceinline__ void ff_butterfly(const int32_t* x, int32_t round, int32_t* a, int32_t* b) {
    const int32_t W1 = 22725, W2 = 21407, W3 = 19265, W4 = 16384, W5 = 12873, W6 = 8867, W7 = 4520;
    const int32_t base = wadd(wmul(W4, x[0]), round);
    a[0] = wadd(wadd(wadd(base, wmul(W2, x[2])), wmul(W4, x[4])), wmul(W6, x[6]));
    a[1] = wsub(wsub(wadd(base, wmul(W6, x[2])), wmul(W4, x[4])), wmul(W2, x[6]));
    a[2] = wadd(wsub(wsub(base, wmul(W6, x[2])), wmul(W4, x[4])), wmul(W2, x[6]));
    a[3] = wsub(wadd(wsub(base, wmul(W2, x[2])), wmul(W4, x[4])), wmul(W6, x[6]));
    b[0] = wadd(wadd(wadd(wmul(W1, x[1]), wmul(W3, x[3])), wmul(W5, x[5])), wmul(W7, x[7]));
    b[1] = wsub(wsub(wsub(wmul(W3, x[1]), wmul(W7, x[3])), wmul(W1, x[5])), wmul(W5, x[7]));
    b[2] = wadd(wadd(wsub(wmul(W5, x[1]), wmul(W1, x[3])), wmul(W7, x[5])), wmul(W3, x[7]));
    b[3] = wsub(wadd(wsub(wmul(W7, x[1]), wmul(W5, x[3])), wmul(W3, x[5])), wmul(W1, x[7]));
}
// Row pass (src/idct.rs:334-338): dequantized int16 in, int32 out.
__device__ __forceinline__ void ffmpeg_row(const int16_t* x16, int32_t* y) {
    int32_t x[8], a[4], b[4];
#pragma unroll
    for (int i = 0; i < 8; i++) x[i] = x16[i];
    ff_butterfly(x, 1 << 12, a, b);
#pragma unroll
    for (int k = 0; k < 4; k++) {
        y[k] = wadd(a[k], b[k]) >> 13;
        y[7 - k] = wsub(a[k], b[k]) >> 13;
    }
}
// Column pass (src/idct.rs:340-351) and code_value (src/idct.rs:263-265).
__device__ __forceinline__ void ffmpeg_col(const int32_t* col, uint16_t* out) {
    int32_t x[8], a[4], b[4];
#pragma unroll
    for (int i = 0; i < 8; i++) x[i] = col[i];
    x[0] = wadd(x[0], 1);
    ff_butterfly(x, 0, a, b);
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const int32_t lo = wadd(a[k], b[k]) >> 15, hi = wsub(a[k], b[k]) >> 15;
        out[k] = uint16_t(min(max(wadd(lo, 32768), 0), 65535));
        out[7 - k] = uint16_t(min(max(wadd(hi, 32768), 0), 65535));
    }
}

// ---------------------------------------------------------------------------
// Linearization curve, src/curve.rs:14-24, from per-segment (c0, delta).
__device__ __forceinline__ uint32_t curve_apply(const uint32_t* c0, const uint32_t* delta, uint32_t code) {
    const uint32_t seg = code >> 13;
    const uint32_t frac = code & 0x1FFF;
    return min((c0[seg] * 8192u + delta[seg] * frac + 4096u) >> 13, 65535u);
}

}  // namespace prr
