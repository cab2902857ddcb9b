// prr_oracle.cpp -- CPU oracle for the ProRes RAW decode / linearize / develop path.
//
// TEST INFRASTRUCTURE ONLY: a C++ restatement of the proresraw_rs crate's CPU
// path, used as the parity checker of the CUDA library and as the timed CPU
// baseline. Every function names the reference file:line it restates.
// Build flags matter: -ffp-contract=off (Rust never contracts a*b+c; fused
// multiply-adds appear only where the crate calls mul_add) and -fwrapv (the
// crate's wrapping integer arithmetic).
//
// Threading follows the crate's rayon decomposition: tile rows for decoding
// (src/decoder.rs:249-254, src/reduced.rs:181-186) and 32-row bands for the
// raw conversion (src/demosaic.rs:306-351).

#include "prr_oracle.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <functional>
#include <thread>
#include <vector>

namespace {

// ---------------------------------------------------------------------------
// Parallel loop over [0, n) on `threads` std::threads (0 = hardware count).
void parallel_for(size_t n, int threads, const std::function<void(size_t)>& f) {
    size_t t = threads > 0 ? size_t(threads) : std::max(1u, std::thread::hardware_concurrency());
    t = std::min(t, n);
    if (t <= 1) {
        for (size_t i = 0; i < n; i++) f(i);
        return;
    }
    std::atomic<size_t> next{0};
    std::vector<std::thread> pool;
    pool.reserve(t);
    for (size_t k = 0; k < t; k++) {
        pool.emplace_back([&] {
            for (size_t i = next.fetch_add(1); i < n; i = next.fetch_add(1)) f(i);
        });
    }
    for (auto& th : pool) th.join();
}

inline uint16_t be16(const uint8_t* p) { return uint16_t(p[0] << 8 | p[1]); }
inline uint32_t be32(const uint8_t* p) {
    return uint32_t(p[0]) << 24 | uint32_t(p[1]) << 16 | uint32_t(p[2]) << 8 | p[3];
}
inline float bef32(const uint8_t* p) {
    uint32_t u = be32(p);
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}

void set_err(orc_error* e, int code) {
    if (e) {
        std::memset(e, 0, sizeof(*e));
        e->code = code;
    }
}
void set_trunc(orc_error* e, const char* what, size_t needed, size_t available) {
    if (e) {
        set_err(e, ORC_ERR_TRUNCATED);
        std::strncpy(e->what, what, sizeof(e->what) - 1);
        e->needed = needed;
        e->available = available;
    }
}

// ---------------------------------------------------------------------------
// codebook.rs:25-110 -- parameters packed (switch << 8) | (exp << 4) | rice.
const uint16_t FIRST_DC = 0x2BC;
const uint16_t DC_RESET = 0x064;
const uint16_t AC_INITIAL = 0x031;
const uint16_t RN_INITIAL = 0x000;
const uint16_t LN_INITIAL = 0x042;
const uint16_t DC_CB[13] = {0x010, 0x021, 0x032, 0x033, 0x033, 0x033, 0x044,
                            0x044, 0x044, 0x044, 0x044, 0x044, 0x076};
const uint16_t RN_CB[28] = {0x200, 0x100, 0x000, 0x000, 0x211, 0x211, 0x111, 0x111, 0x011, 0x011,
                            0x021, 0x021, 0x222, 0x022, 0x022, 0x022, 0x022, 0x022, 0x022, 0x022,
                            0x022, 0x022, 0x022, 0x022, 0x022, 0x032, 0x032, 0x044};
const uint16_t LN_CB[15] = {0x100, 0x111, 0x222, 0x222, 0x122, 0x122, 0x433, 0x433,
                            0x233, 0x233, 0x233, 0x233, 0x233, 0x233, 0x033};
struct AcTable {
    uint16_t t[95];
    AcTable() {
        // codebook.rs:57-85: runs of equal entries.
        const int counts[10] = {1, 1, 2, 3, 3, 8, 2, 22, 52, 1};
        const uint16_t vals[10] = {0x000, 0x211, 0x111, 0x222, 0x122,
                                   0x233, 0x133, 0x244, 0x355, 0x166};
        int i = 0;
        for (int r = 0; r < 10; r++)
            for (int k = 0; k < counts[r]; k++) t[i++] = vals[r];
    }
};
const AcTable AC_CB;
const uint8_t SCAN[64] = {0,  8,  1,  9,  16, 24, 17, 25, 2,  10, 3,  11, 18, 26, 19, 27,
                          32, 40, 33, 34, 41, 48, 56, 49, 42, 35, 43, 50, 57, 58, 51, 59,
                          4,  12, 5,  6,  13, 20, 28, 21, 14, 7,  15, 22, 29, 36, 44, 37,
                          30, 23, 31, 38, 45, 52, 60, 53, 46, 39, 47, 54, 61, 62, 55, 63};
const uint8_t SCAN_4X4[16] = {0, 4, 1, 5, 8, 12, 9, 13, 2, 6, 3, 7, 10, 14, 11, 15};
const uint8_t SCAN_2X2[4] = {0, 2, 1, 3};

inline uint16_t next_cb(const uint16_t* table, size_t n, uint32_t symbol) {
    return table[std::min<size_t>(symbol, n - 1)];  // coefficients.rs:16-18
}

// ---------------------------------------------------------------------------
// bits.rs:17-134 -- 64-bit window reader.
uint32_t partial_word(const uint8_t* b, size_t n) {  // bits.rs:31-37
    uint32_t w = 0;
    for (size_t i = 0; i < n && i < 4; i++) w |= uint32_t(b[i]) << (24 - 8 * i);
    return w;
}

struct BitReader {
    const uint8_t* data;
    size_t len;
    size_t pos;
    size_t words_end;
    uint64_t window;
    int32_t extra;

    BitReader(const uint8_t* d, size_t n, size_t align) : data(d), len(n) {  // bits.rs:44-76
        size_t remaining = n;
        size_t address = align;
        uint32_t first;
        if (remaining < 4) {
            first = partial_word(d, remaining);
            pos = remaining;
            address += remaining;
            remaining = 0;
        } else {
            first = be32(d);
            pos = 4;
            address += 4;
            remaining -= 4;
        }
        uint32_t low = 0;
        extra = 0;
        size_t to_boundary = (4 - (address & 3)) & 3;
        if (to_boundary != 0 && to_boundary <= remaining) {
            low = partial_word(d + pos, to_boundary);
            pos += to_boundary;
            remaining -= to_boundary;
            extra = int32_t(8 * to_boundary);
        }
        words_end = pos + 4 * (remaining / 4);
        window = (uint64_t(first) << 32) | uint64_t(low);
    }
    uint32_t next_word() {  // bits.rs:79-89
        if (pos < words_end) {
            uint32_t w = be32(data + pos);
            pos += 4;
            return w;
        }
        uint32_t w = partial_word(data + pos, len - pos);
        pos = len;
        return w;
    }
    uint32_t top() const { return uint32_t(window >> 32); }
    void consume(uint32_t n) {  // bits.rs:97-105
        window = window << (n & 63);
        extra = int32_t(uint32_t(extra) - n);
        if (extra < 0) {
            uint32_t shift = uint32_t(-int32_t(int8_t(extra))) & 0x3f;
            window |= uint64_t(next_word()) << shift;
            extra += 32;
        }
    }
};

// bits.rs:116-134
inline void codeword(uint32_t p, uint16_t cb, uint32_t& value, uint32_t& len) {
    uint32_t lz = uint32_t(__builtin_clz(p));
    uint32_t s = cb >> 8;
    uint32_t r = cb & 0xF;
    if (int32_t(p) < 0) {
        value = (p & 0x7fffffffu) >> ((31u - r) & 31);
        len = r + 1;
        return;
    }
    if (lz <= s) {
        uint32_t tail = ((p << ((lz + 1) & 31)) >> 1) >> ((31u - r) & 31);
        value = (lz << r) + tail;
        len = r + 1 + lz;
        return;
    }
    uint32_t e = (cb >> 4) & 0xF;
    len = 2 * lz - s + e;
    value = ((s + 1) << r) + (p >> ((32u - len) & 31)) - (1u << e);
}

// coefficients.rs:37-146
void decode_component_reduced(const uint8_t* data, size_t len, size_t align, uint32_t log2_blocks,
                              uint32_t log2_coefs, int16_t* coefs) {
    const uint8_t* scan = log2_coefs == 6 ? SCAN : log2_coefs == 4 ? SCAN_4X4 : SCAN_2X2;
    const uint32_t per_block = 1u << log2_coefs;
    const uint32_t blocks = 1u << log2_blocks;
    const uint32_t codes = per_block * blocks;
    const uint32_t block_mask = blocks - 1;
    std::memset(coefs, 0, sizeof(int16_t) * codes);
    BitReader r(data, len, align);
    if (r.top() == 0) return;
    uint32_t first, l;
    codeword(r.top(), FIRST_DC, first, l);
    r.consume(l);
    uint32_t odd = first & 1;
    int32_t dc = int32_t((((odd + first) >> 1) ^ (0u - odd)) + odd);
    coefs[0] = int16_t(dc);
    uint16_t dc_cb = DC_RESET;
    uint32_t sign = 0;
    for (uint32_t block = 1; block < blocks; block++) {
        if (r.top() == 0) return;
        uint32_t symbol;
        codeword(r.top(), dc_cb, symbol, l);
        sign ^= symbol & 1;
        uint32_t magnitude = ((symbol & 1) + symbol) >> 1;
        int32_t delta = int32_t(((0u - sign) ^ magnitude) + sign);
        dc_cb = next_cb(DC_CB, 13, magnitude);
        sign = delta < 0 ? 1 : 0;
        r.consume(l);
        dc = int32_t(uint32_t(dc) + uint32_t(delta));
        coefs[per_block * block] = int16_t(dc);
    }
    auto place = [&](uint32_t n) -> size_t {
        return size_t(scan[n >> log2_blocks]) + size_t((n & block_mask) << log2_coefs);
    };
    auto level = [&](uint16_t cb, uint32_t& symbol) -> int16_t {
        uint32_t top = r.top();
        uint32_t ln;
        codeword(top, cb, symbol, ln);
        bool negative = ((int32_t(top << (ln & 31))) >> 31) != 0;
        r.consume(ln + 1);
        uint16_t magnitude = uint16_t(uint16_t(symbol) + 1);
        return int16_t(negative ? uint16_t(0u - magnitude) : magnitude);
    };
    uint16_t ac_cb = AC_INITIAL, rn_cb = RN_INITIAL, ln_cb = LN_INITIAL;
    uint32_t n = blocks;
    if (n >= codes) return;
    while (r.top() != 0) {
        uint32_t run;
        codeword(r.top(), ln_cb, run, l);
        r.consume(l);
        for (uint32_t i = 0; i < run; i++) {
            if (r.top() == 0) return;
            uint32_t symbol;
            int16_t v = level(ac_cb, symbol);
            ac_cb = next_cb(AC_CB.t, 95, symbol);
            coefs[place(n)] = v;
            n += 1;
            if (n == codes) return;
        }
        if (r.top() == 0) return;
        uint32_t zeros;
        codeword(r.top(), rn_cb, zeros, l);
        rn_cb = next_cb(RN_CB, 28, zeros);
        r.consume(l);
        n = n + 1 + zeros;
        if (n >= codes || r.top() == 0) return;
        uint32_t symbol;
        int16_t v = level(ac_cb, symbol);
        ac_cb = next_cb(AC_CB.t, 95, symbol);
        ln_cb = next_cb(LN_CB, 15, symbol);
        coefs[place(n)] = v;
        n += 1;
        if (n >= codes) return;
    }
}

// ---------------------------------------------------------------------------
// idct.rs:39-351
inline int16_t dequantize(int16_t coef, int16_t q) {  // idct.rs:41-43
    int32_t v = int32_t(coef) * int32_t(q);
    return int16_t(std::clamp(v, -32768, 32767));
}

const int32_t ROW_TABLES[4][4][8] = {  // idct.rs:51-76
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
const int ROW_SET[8] = {0, 1, 2, 3, 0, 3, 2, 1};

inline float f32_bits(uint32_t u) {
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}
const float SCALE = f32_bits(0x39800000u);  // 2^-12
const float BIAS = f32_bits(0x47000080u);   // 32768.5
const float TAN1 = f32_bits(0x3e4bafafu);
const float TAN2 = f32_bits(0x3ed413cdu);
const float TAN3 = f32_bits(0x3f2b0dc1u);
const float COS4 = f32_bits(0x3f3504f3u);
const float SCALE4 = f32_bits(0x39000000u);  // 2^-13

void row_pass(const int16_t* x16, const int32_t (*t)[8], int32_t* out) {  // idct.rs:93-105
    int32_t x[8];
    for (int i = 0; i < 8; i++) x[i] = x16[i];
    const int32_t pa[4] = {x[0], x[4], x[1], x[5]};
    const int32_t pb[4] = {x[2], x[6], x[3], x[7]};
    for (int k = 0; k < 4; k++) {
        auto dot = [&](int j) { return pa[j] * t[j][2 * k] + pb[j] * t[j][2 * k + 1]; };
        int32_t even = dot(0) + dot(1);
        int32_t odd = dot(2) + dot(3);
        out[k] = even + odd;
        out[7 - k] = even - odd;
    }
}

inline int32_t trunc_to_i32(float v) {  // idct.rs:109-115
    if (v >= -2147483648.0f && v < 2147483648.0f) return int32_t(v);
    return INT32_MIN;
}
inline uint16_t output_code(float v) {  // idct.rs:120-123
    int32_t centred = std::clamp(int32_t(uint32_t(trunc_to_i32(v)) - 32768u), -32768, 32767);
    return uint16_t(uint16_t(int16_t(centred)) ^ 0x8000);
}

void apple_block(const int16_t* coefs, const int16_t* q, uint16_t* out) {  // idct.rs:126-174
    float rows[8][8];
    for (int r = 0; r < 8; r++) {
        int16_t d[8];
        for (int c = 0; c < 8; c++) d[c] = dequantize(coefs[8 * r + c], q[8 * r + c]);
        int32_t y[8];
        row_pass(d, ROW_TABLES[ROW_SET[r]], y);
        for (int c = 0; c < 8; c++) rows[r][c] = float(y[c]) * SCALE;
    }
    for (int c = 0; c < 8; c++) {
        float r[8];
        for (int i = 0; i < 8; i++) r[i] = rows[i][c];
        float p = r[0] + BIAS;
        float ea = p + r[4];
        float eb = p - r[4];
        float f = r[6] * TAN2 + r[2];
        float g = r[2] * TAN2 - r[6];
        float e0 = ea + f, e3 = ea - f, e1 = eb + g, e2 = eb - g;
        float a = r[7] * TAN1 + r[1];
        float b = r[1] * TAN1 - r[7];
        float cc = r[5] * TAN3 + r[3];
        float d = r[5] - r[3] * TAN3;
        float o0 = a + cc, t = a - cc, o3 = b + d, u = b - d;
        float o1 = (t + u) * COS4;
        float o2 = (t - u) * COS4;
        float y[8] = {e0 + o0, e1 + o1, e2 + o2, e3 + o3, e3 - o3, e2 - o2, e1 - o1, e0 - o0};
        for (int i = 0; i < 8; i++) out[8 * i + c] = output_code(y[i]);
    }
}

const int32_t ROW4_K[2] = {8192, 10703};  // idct.rs:179-182
const int32_t ROW4_T[2][4] = {{10703, 4433, 4433, -10703}, {13985, 5793, 5793, -13985}};

inline uint16_t saturate_code(int32_t v) {  // idct.rs:189-191
    return uint16_t(uint16_t(int16_t(std::clamp(v, -32768, 32767))) ^ 0x8000);
}

void apple_block_4x4(const int16_t* coefs, const int16_t* q, uint16_t* out) {  // idct.rs:197-226
    float rows[4][4];
    for (int r = 0; r < 4; r++) {
        int32_t x[4];
        for (int c = 0; c < 4; c++) x[c] = dequantize(coefs[4 * r + c], q[8 * r + c]);
        int32_t k = ROW4_K[r & 1];
        const int32_t* t = ROW4_T[r & 1];
        int32_t e0 = k * x[0] + k * x[2];
        int32_t e1 = k * x[0] - k * x[2];
        int32_t o0 = t[0] * x[1] + t[1] * x[3];
        int32_t o1 = t[2] * x[1] + t[3] * x[3];
        int32_t y[4] = {e0 + o0, e1 + o1, e1 - o1, e0 - o0};
        for (int c = 0; c < 4; c++) rows[r][c] = float(y[c]) * SCALE4;
    }
    for (int c = 0; c < 4; c++) {
        float r0 = rows[0][c] + BIAS;
        float r1 = rows[1][c], r2 = rows[2][c], r3 = rows[3][c];
        float e0 = r2 + r0;
        float e1 = r0 - r2;
        float f = r3 * TAN2 + r1;
        float g = r1 * TAN2 - r3;
        float y[4] = {f + e0, g + e1, e1 - g, e0 - f};
        for (int i = 0; i < 4; i++) out[4 * i + c] = output_code(y[i]);
    }
}

void apple_block_2x2(const int16_t* coefs, const int16_t* q, uint16_t* out) {  // idct.rs:232-247
    int32_t d0 = dequantize(coefs[0], q[0]);
    int32_t d1 = dequantize(coefs[1], q[1]);
    int32_t d2 = dequantize(coefs[2], q[8]);
    int32_t d3 = dequantize(coefs[3], q[9]);
    int32_t ts = d0 + d1, td = d0 - d1, bs = d2 + d3, bd = d2 - d3;
    out[0] = saturate_code(ts + bs);
    out[1] = saturate_code(td + bd);
    out[2] = saturate_code(ts - bs);
    out[3] = saturate_code(td - bd);
}

// FFmpeg simple IDCT, idct.rs:252-351 (wrapping 32-bit arithmetic; -fwrapv).
const int32_t W1 = 22725, W2 = 21407, W3 = 19265, W4 = 16384, W5 = 12873, W6 = 8867, W7 = 4520;

inline uint16_t code_value(int32_t centered) {  // idct.rs:263-265
    return uint16_t(std::clamp(centered + 32768, 0, 65535));
}

void butterfly(const int32_t* x, int32_t round, int32_t* a, int32_t* b) {  // idct.rs:282-318
    int32_t base = W4 * x[0] + round;
    a[0] = base + W2 * x[2] + W4 * x[4] + W6 * x[6];
    a[1] = base + W6 * x[2] - W4 * x[4] - W2 * x[6];
    a[2] = base - W6 * x[2] - W4 * x[4] + W2 * x[6];
    a[3] = base - W2 * x[2] + W4 * x[4] - W6 * x[6];
    b[0] = W1 * x[1] + W3 * x[3] + W5 * x[5] + W7 * x[7];
    b[1] = W3 * x[1] - W7 * x[3] - W1 * x[5] - W5 * x[7];
    b[2] = W5 * x[1] - W1 * x[3] + W7 * x[5] + W3 * x[7];
    b[3] = W7 * x[1] - W5 * x[3] + W3 * x[5] - W1 * x[7];
}

void ffmpeg_block(const int16_t* coefs, const int16_t* q, uint16_t* out) {  // idct.rs:268-277
    int32_t blk[64];
    for (int i = 0; i < 64; i++) blk[i] = dequantize(coefs[i], q[i]);
    for (int r = 0; r < 8; r++) {  // idct.rs:334-338
        int32_t a[4], b[4];
        butterfly(blk + 8 * r, 1 << 12, a, b);
        int32_t* y = blk + 8 * r;
        y[0] = (a[0] + b[0]) >> 13;
        y[1] = (a[1] + b[1]) >> 13;
        y[2] = (a[2] + b[2]) >> 13;
        y[3] = (a[3] + b[3]) >> 13;
        y[4] = (a[3] - b[3]) >> 13;
        y[5] = (a[2] - b[2]) >> 13;
        y[6] = (a[1] - b[1]) >> 13;
        y[7] = (a[0] - b[0]) >> 13;
    }
    for (int c = 0; c < 8; c++) {  // idct.rs:340-351
        int32_t x[8], a[4], b[4];
        for (int i = 0; i < 8; i++) x[i] = blk[8 * i + c];
        x[0] = x[0] + 1;
        butterfly(x, 0, a, b);
        int32_t y[8] = {(a[0] + b[0]) >> 15, (a[1] + b[1]) >> 15, (a[2] + b[2]) >> 15,
                        (a[3] + b[3]) >> 15, (a[3] - b[3]) >> 15, (a[2] - b[2]) >> 15,
                        (a[1] - b[1]) >> 15, (a[0] - b[0]) >> 15};
        for (int i = 0; i < 8; i++) blk[8 * i + c] = y[i];
    }
    for (int i = 0; i < 64; i++) out[i] = code_value(blk[i]);
}

// ---------------------------------------------------------------------------
// curve.rs:14-33
inline uint16_t curve_linearize(const uint16_t* curve, uint16_t code) {
    uint32_t seg = code >> 13;
    uint32_t frac = code & 0x1FFF;
    uint32_t c0 = curve[seg];
    uint32_t c1 = seg + 1 < 8 ? curve[seg + 1] : 65536u;
    uint32_t delta = (c1 - c0) & 0xFFFF;
    uint32_t out = (c0 * 8192 + delta * frac + 4096) >> 13;
    return uint16_t(std::min<uint32_t>(out, 65535));
}
std::vector<uint16_t> curve_lut(const uint16_t* curve) {
    std::vector<uint16_t> lut(65536);
    for (uint32_t c = 0; c < 65536; c++) lut[c] = curve_linearize(curve, uint16_t(c));
    return lut;
}

// ---------------------------------------------------------------------------
// header.rs:156-246, decoder.rs:45-123, tile.rs:36-153
const size_t PREFIX_LEN = 10;
const size_t FIXED_BODY_LEN = 70;
const uint16_t MIN_HEADER_SIZE = 72;
const uint16_t DEFAULT_CURVE[8] = {0, 512, 1024, 2048, 4096, 8192, 16384, 32768};

int header_parse_body(const uint8_t* body, size_t n, orc_header* h, orc_error* err) {
    if (n < FIXED_BODY_LEN) {
        set_trunc(err, "frame header", FIXED_BODY_LEN, n);
        return ORC_ERR_TRUNCATED;
    }
    std::memset(h, 0, sizeof(*h));
    h->version = body[1];
    if (h->version > 1) {
        set_err(err, ORC_ERR_UNSUPPORTED_VERSION);
        if (err) err->value = h->version;
        return ORC_ERR_UNSUPPORTED_VERSION;
    }
    std::memcpy(h->vendor, body + 2, 4);
    h->width = be16(body + 6);
    h->height = be16(body + 8);
    if (h->width == 0 || h->height == 0 || (h->width & 1) || (h->height & 1)) {
        set_err(err, ORC_ERR_BAD_DIMENSIONS);
        if (err) {
            err->width = h->width;
            err->height = h->height;
        }
        return ORC_ERR_BAD_DIMENSIONS;
    }
    std::memcpy(h->crop, body + 10, 4);
    h->bayer_pattern = uint8_t(be16(body + 14) & 3);
    h->white_level = uint16_t(be16(body + 16) + 256);
    h->wb_red = bef32(body + 18);
    h->wb_blue = bef32(body + 22);
    for (int i = 0; i < 9; i++) h->color_matrix[i] = bef32(body + 26 + 4 * i);
    h->gain = bef32(body + 62);
    h->wb_cct = be16(body + 66);
    h->flags = be16(body + 68);
    h->alignment = uint8_t((h->flags >> 1) & 7);
    if (h->alignment > 4) {
        set_err(err, ORC_ERR_BAD_ALIGNMENT);
        if (err) err->value = h->alignment;
        return ORC_ERR_BAD_ALIGNMENT;
    }
    size_t pos = FIXED_BODY_LEN;
    std::fill(h->quant_matrix, h->quant_matrix + 64, 1);
    if (h->flags & 1) {
        if (pos + 64 > n) {
            set_trunc(err, "quantization matrix", pos + 64, n);
            return ORC_ERR_TRUNCATED;
        }
        std::memcpy(h->quant_matrix, body + pos, 64);
        pos += 64;
        for (int i = 0; i < 64; i++) {
            if (h->quant_matrix[i] < 1 || h->quant_matrix[i] > 63) {
                set_err(err, ORC_ERR_BAD_QUANT_MATRIX);
                if (err) {
                    err->index = i;
                    err->value = h->quant_matrix[i];
                }
                return ORC_ERR_BAD_QUANT_MATRIX;
            }
        }
    }
    if ((h->flags >> 4) & 1) {
        if (pos + 16 > n) {
            set_trunc(err, "linearization curve", pos + 16, n);
            return ORC_ERR_TRUNCATED;
        }
        uint16_t pts[8];
        for (int i = 0; i < 8; i++) pts[i] = be16(body + pos + 2 * i);
        if (h->version == 0) {
            set_err(err, ORC_ERR_UNEXPECTED_CURVE);
            return ORC_ERR_UNEXPECTED_CURVE;
        }
        for (int i = 0; i < 7; i++) {
            if (pts[i] >= pts[i + 1]) {
                set_err(err, ORC_ERR_BAD_CURVE);
                if (err) std::memcpy(err->curve, pts, sizeof(pts));
                return ORC_ERR_BAD_CURVE;
            }
        }
        std::memcpy(h->curve, pts, sizeof(pts));
    } else {
        std::memcpy(h->curve, DEFAULT_CURVE, sizeof(DEFAULT_CURVE));
    }
    return ORC_OK;
}

int header_len(const uint8_t* pkt, size_t len, size_t* out, orc_error* err) {  // decoder.rs:58-73
    if (len < PREFIX_LEN) {
        set_trunc(err, "frame prefix", PREFIX_LEN, len);
        return ORC_ERR_TRUNCATED;
    }
    if (std::memcmp(pkt + 4, "prrf", 4) != 0) {
        set_err(err, ORC_ERR_BAD_TAG);
        if (err) std::memcpy(err->tag, pkt + 4, 4);
        return ORC_ERR_BAD_TAG;
    }
    uint16_t hs = be16(pkt + 8);
    if (hs < MIN_HEADER_SIZE) {
        set_err(err, ORC_ERR_HEADER_TOO_SHORT);
        if (err) err->value = hs;
        return ORC_ERR_HEADER_TOO_SHORT;
    }
    *out = PREFIX_LEN + size_t(hs) - 2;
    return ORC_OK;
}

int parse_header(const uint8_t* pkt, size_t len, orc_header* h, orc_error* err) {  // decoder.rs:45-53
    size_t body_end;
    int rc = header_len(pkt, len, &body_end, err);
    if (rc) return rc;
    if (body_end > len) {
        set_trunc(err, "frame header", body_end, len);
        return ORC_ERR_TRUNCATED;
    }
    return header_parse_body(pkt + PREFIX_LEN, body_end - PREFIX_LEN, h, err);
}

struct Geometry {
    size_t x;
    uint32_t log2;
};
struct Grid {  // tile.rs:36-107
    size_t columns, rows;
    uint32_t alignment;
    Grid(size_t w, size_t h, uint32_t a) : columns((w + 15) / 16), rows((h + 15) / 16), alignment(a) {}
    size_t tiles_per_row() const {
        size_t full = columns >> alignment;
        size_t rem = columns & ((size_t(1) << alignment) - 1);
        return full + size_t(__builtin_popcountll(rem));
    }
    size_t len() const { return tiles_per_row() * rows; }
    std::vector<Geometry> row() const {
        std::vector<Geometry> out;
        size_t column = 0, remaining = columns;
        uint32_t log2 = alignment;
        while (remaining > 0) {
            size_t unit = size_t(1) << log2;
            if (unit <= remaining) {
                out.push_back({column * 16, log2});
                column += unit;
                remaining -= unit;
            } else {
                log2 -= 1;
            }
        }
        return out;
    }
};

struct Parsed {
    orc_header header;
    size_t tiles_per_row, rows;
    std::vector<size_t> off, len;
    uint8_t max_qscale;
};

int parse_frame(const uint8_t* pkt, size_t len, Parsed& p, orc_error* err) {  // decoder.rs:76-123
    if (len < PREFIX_LEN) {
        set_trunc(err, "frame prefix", PREFIX_LEN, len);
        return ORC_ERR_TRUNCATED;
    }
    uint32_t declared = be32(pkt);
    if (declared == 0 || size_t(declared) > len) {
        set_err(err, ORC_ERR_FRAME_SIZE_MISMATCH);
        if (err) {
            err->declared = declared;
            err->actual = len;
        }
        return ORC_ERR_FRAME_SIZE_MISMATCH;
    }
    size_t body_end;
    int rc = header_len(pkt, len, &body_end, err);
    if (rc) return rc;
    rc = parse_header(pkt, len, &p.header, err);
    if (rc) return rc;
    Grid grid(p.header.width, p.header.height, p.header.alignment);
    size_t ntiles = grid.len();
    size_t table_end = body_end + 2 * ntiles;
    if (table_end > len) {
        set_trunc(err, "tile size table", table_end, len);
        return ORC_ERR_TRUNCATED;
    }
    p.tiles_per_row = grid.tiles_per_row();
    p.rows = grid.rows;
    p.off.resize(ntiles);
    p.len.resize(ntiles);
    size_t offset = table_end;
    uint8_t maxq = 0;
    for (size_t i = 0; i < ntiles; i++) {
        size_t size = be16(pkt + body_end + 2 * i);
        uint8_t qb = offset + 1 < len ? pkt[offset + 1] : 0;
        maxq = std::max(maxq, qb);
        if (offset + size > len) {
            set_err(err, ORC_ERR_TILE_OUT_OF_BOUNDS);
            if (err) err->index = i;
            return ORC_ERR_TILE_OUT_OF_BOUNDS;
        }
        p.off[i] = offset;
        p.len[i] = size;
        offset += size;
    }
    p.max_qscale = maxq;
    return ORC_OK;
}

struct Tile {
    uint8_t qscale;
    size_t soff[4], slen[4];  // relative to the tile start
};
bool tile_parse(const uint8_t* d, size_t len, Tile& t) {  // tile.rs:126-153
    if (len < 8) return false;
    size_t header_len = d[0] >> 3;
    uint8_t qscale = d[1];
    size_t sizes[3] = {be16(d + 2), be16(d + 4), be16(d + 6)};
    if (header_len < 8 || qscale == 0 || sizes[0] == 0 || sizes[1] == 0 || sizes[2] == 0)
        return false;
    size_t used = header_len + sizes[0] + sizes[1] + sizes[2];
    if (used >= len) return false;
    t.qscale = qscale;
    size_t o = header_len;
    for (int s = 0; s < 3; s++) {
        t.soff[s] = o;
        t.slen[s] = sizes[s];
        o += sizes[s];
    }
    t.soff[3] = o;
    t.slen[3] = len - o;
    return true;
}

// header.rs:64-82: stream s lands on phase (row, col).
void stream_phases(uint8_t pattern, int ph[4][2]) {
    int r = (pattern == 2 || pattern == 3) ? 1 : 0;
    int c = (pattern == 1 || pattern == 3) ? 1 : 0;
    ph[0][0] = 1 - r; ph[0][1] = c;
    ph[1][0] = r;     ph[1][1] = 1 - c;
    ph[2][0] = 1 - r; ph[2][1] = 1 - c;
    ph[3][0] = r;     ph[3][1] = c;
}

// decoder.rs:272-307
void decode_tile(const uint8_t* pkt, size_t tile_off, const Tile& t, const Geometry& g,
                 const uint8_t* qmat, const int ph[4][2], int idct, uint16_t* rows,
                 size_t stride) {
    int16_t scaled[64];
    for (int i = 0; i < 64; i++) scaled[i] = int16_t(uint16_t(qmat[i]) * uint16_t(t.qscale));
    size_t blocks = size_t(1) << g.log2;
    int16_t coefs[64 * 16];
    for (int s = 0; s < 4; s++) {
        size_t off = tile_off + t.soff[s];
        decode_component_reduced(pkt + off, t.slen[s], off & 3, g.log2, 6, coefs);
        for (size_t b = 0; b < blocks; b++) {
            uint16_t values[64];
            if (idct == 0)
                apple_block(coefs + 64 * b, scaled, values);
            else
                ffmpeg_block(coefs + 64 * b, scaled, values);
            size_t x0 = g.x + b * 16 + ph[s][1];
            for (int i = 0; i < 8; i++) {
                uint16_t* dst = rows + (2 * i + ph[s][0]) * stride + x0;
                for (int j = 0; j < 8; j++) dst[2 * j] = values[8 * i + j];
            }
        }
    }
}

// ---------------------------------------------------------------------------
// demosaic.rs
const double XYZ_TO_REC2020[3][3] = {  // demosaic.rs:37-41
    {1.716651187971268, -0.355670783776393, -0.25336628137366},
    {-0.666684351832489, 1.616481236634939, 0.015768545813911},
    {0.017639857445311, -0.042770613257809, 0.942103121235474}};

inline float fma32(float a, float b, float c) { return std::fma(a, b, c); }

inline float variance(float v, float off, const float* n) {  // demosaic.rs:423-426
    float t = off + v;
    return n[2] + std::max(n[1], n[0] * (t * t));
}
inline float dot4(const float* a, const float* b) {  // demosaic.rs:431-433
    return fma32(a[3], b[3], fma32(a[2], b[2], fma32(a[0], b[0], a[1] * b[1])));
}
inline void mirror(float* d, size_t pos, size_t len, float c) {  // demosaic.rs:547-557
    if (pos == 0) {
        float d1 = d[1], d3 = d[3];
        d[0] = d1; d[1] = d1; d[2] = d3; d[3] = d3;
    } else if (pos == 1) {
        d[2] = c;
    } else if (pos == len - 1) {
        float d0 = d[0], d2 = d[2];
        d[0] = d0; d[1] = d0; d[2] = d2; d[3] = d2;
    } else if (pos == len - 2) {
        d[3] = c;
    }
}
inline void mirrored(size_t y, size_t len, size_t& ym, size_t& yp) {  // demosaic.rs:406-411
    ym = y > 0 ? y - 1 : y + 1;
    yp = y < len - 1 ? y + 1 : y - 1;
}

// demosaic.rs:481-541
void green_row(const float* const rows[5], size_t y, size_t h, size_t w, const orc_params& p,
               float* out /* 2*w */) {
    const float bs = float(p.black) * p.one_over_range;
    const size_t red_row = size_t(p.cfa_phase >> 1);
    const size_t red_col = size_t(p.cfa_phase & 1);
    const size_t last_x = w - 1;
    const float* centre = rows[2];
    for (size_t x = 0; x < w; x++) {
        out[2 * x] = 0.0f;
        out[2 * x + 1] = centre[x];
    }
    const bool phase = (y % 2) == red_row;
    const size_t first = phase ? red_col : 1 - red_col;
    const float clip = phase ? p.clip[0] : p.clip[1];
    const float limit[4] = {1.0f, 1.0f, clip, clip};
    auto var = [&](float v) { return variance(v, bs, p.noise); };
    for (size_t x = first; x < w; x += 2) {
        float c = std::min(centre[x], clip);
        auto at = [&](long dx) {
            long i = std::clamp(long(x) + dx, 0L, long(last_x));
            return centre[i];
        };
        float hh[4] = {at(-1), at(1), at(-2), at(2)};
        float vv[4] = {rows[1][x], rows[3][x], rows[0][x], rows[4][x]};
        for (int i = 0; i < 4; i++) {
            hh[i] = std::min(hh[i], limit[i]);
            vv[i] = std::min(vv[i], limit[i]);
        }
        mirror(hh, x, w, c);
        mirror(vv, y, h, c);
        float var_h[4], var_v[4];
        for (int i = 0; i < 4; i++) {
            var_h[i] = var(hh[i]);
            var_v[i] = var(vv[i]);
        }
        float sums[4] = {hh[0] + hh[1], vv[0] + vv[1], hh[2] + hh[3], vv[2] + vv[3]};
        float ratio[2] = {0.0f, 0.0f};
        if (c > std::sqrt(var(c))) {
            float t[4] = {c * 2.0f + sums[2], c * 2.0f + sums[3], c * -2.0f + sums[2],
                          c * -2.0f + sums[3]};
            for (int dir = 0; dir < 2; dir++) {
                const float* d = dir == 0 ? hh : vv;
                const float* vd = dir == 0 ? var_h : var_v;
                float sd[4];
                for (int i = 0; i < 4; i++) sd[i] = std::sqrt(vd[i]);
                float a = d[0] - d[1];
                float b = d[2] - d[3];
                bool any = a * b > 0.0f || (d[2] - c) * (d[3] - c) > 0.0f ||
                           sd[0] + sd[1] > std::fabs(a) || sd[2] + sd[3] > std::fabs(b);
                bool all = d[0] > sd[0] && d[1] > sd[1] && d[2] > sd[2] && d[3] > sd[3];
                if (any && all) ratio[dir] = t[2 + dir] / (t[dir] * 2.0f);
            }
        }
        float gh = sums[0] * 0.5f * (1.0f - ratio[0]);
        float gv = sums[1] * 0.5f * (1.0f - ratio[1]);
        float dh[4] = {hh[0] - gh, hh[1] - gh, hh[2] - c, hh[3] - c};
        float dv[4] = {vv[0] - gv, vv[1] - gv, vv[2] - c, vv[3] - c};
        float eh = dot4(dh, dh) + (var_h[0] + var_h[1]);
        float ev = dot4(dv, dv) + (var_v[0] + var_v[1]);
        out[2 * x] = c;
        out[2 * x + 1] = gv + (gh - gv) * ev / (eh + ev);
    }
}

struct Centre {
    float g, sigma;
};

// demosaic.rs:572-604
float estimate(const float xx[4], const float gg[4], Centre c, float off, const float* noise) {
    const float quarter[4] = {0.25f, 0.25f, 0.25f, 0.25f};
    const float ones[4] = {1.0f, 1.0f, 1.0f, 1.0f};
    float mean_x = dot4(xx, quarter);
    if (!(c.sigma < c.g)) return mean_x;
    float var_x[4], sx[4], sg[4];
    for (int i = 0; i < 4; i++) {
        var_x[i] = variance(xx[i], off, noise);
        sx[i] = std::sqrt(var_x[i]);
        sg[i] = std::sqrt(variance(gg[i], off, noise));
    }
    bool above = true;
    for (int i = 0; i < 4; i++) above = above & (sx[i] < xx[i]) & (sg[i] < gg[i]);
    if (!above) return mean_x;
    float cg = c.g, cs = c.sigma;
    float lo[4], mid[4], hi[4];
    for (int i = 0; i < 4; i++) lo[i] = ((cg - cs) * (xx[i] - sx[i])) / (sg[i] + gg[i]);
    for (int i = 0; i < 4; i++) mid[i] = (cg * xx[i]) / gg[i];
    for (int i = 0; i < 4; i++) hi[i] = ((cs + cg) * (sx[i] + xx[i])) / (gg[i] - sg[i]);
    float ml[4], hm[4];
    for (int i = 0; i < 4; i++) {
        ml[i] = mid[i] - lo[i];
        hm[i] = hi[i] - mid[i];
    }
    float spread = dot4(ml, hm);
    float mean_mid = dot4(mid, quarter);
    float dm[4], dx[4];
    for (int i = 0; i < 4; i++) dm[i] = mid[i] - mean_mid;
    float b = fma32(spread, 0.75f, dot4(dm, dm));
    for (int i = 0; i < 4; i++) dx[i] = xx[i] - mean_x;
    float a = fma32(dot4(var_x, ones), 0.75f, dot4(dx, dx));
    float weight = a / (b + a);
    return fma32(mean_mid - mean_x, weight, mean_x);
}

// demosaic.rs:648-688; put(x, rgb)
template <class Put>
void chroma_row(const float* up, const float* mid, const float* down, size_t w, size_t y,
                const orc_params& p, Put put) {
    const float off = p.black_over_range;
    const bool on_red_row = (y % 2) == size_t(p.cfa_phase >> 1);
    const size_t red_col = size_t(p.cfa_phase & 1);
    const size_t rb_col = on_red_row ? red_col : 1 - red_col;
    for (size_t x = 0; x < w; x++) {
        size_t xm, xp;
        mirrored(x, w, xm, xp);
        float c = mid[2 * x], g = mid[2 * x + 1];
        Centre centre{g, std::sqrt(variance(g, off, p.noise))};
        float r, b;
        if (x % 2 == rb_col) {
            const float* n[4] = {up + 2 * xm, down + 2 * xm, up + 2 * xp, down + 2 * xp};
            float xx[4], gg[4];
            for (int i = 0; i < 4; i++) {
                xx[i] = n[i][0];
                gg[i] = n[i][1];
            }
            float e = estimate(xx, gg, centre, off, p.noise);
            if (on_red_row) {
                r = c; b = e;
            } else {
                r = e; b = c;
            }
        } else {
            auto pair = [&](const float* u, const float* v) {
                float xx[4] = {u[0], v[0], u[0], v[0]};
                float gg[4] = {u[1], v[1], u[1], v[1]};
                return estimate(xx, gg, centre, off, p.noise);
            };
            float eh = pair(mid + 2 * xm, mid + 2 * xp);
            float ev = pair(up + 2 * x, down + 2 * x);
            if (on_red_row) {
                r = eh; b = ev;
            } else {
                r = ev; b = eh;
            }
        }
        put(x, std::min(r * p.wb[0], 1.0f), std::min(g, 1.0f), std::min(b * p.wb[1], 1.0f));
    }
}

inline void matrix_px(float& r, float& g, float& b, const float* m) {  // demosaic.rs:700-720
    float rv = r, gv = g, bv = b;
    r = fma32(bv, m[2], fma32(rv, m[0], gv * m[1]));
    g = fma32(bv, m[5], fma32(rv, m[3], gv * m[4]));
    b = fma32(bv, m[8], fma32(rv, m[6], gv * m[7]));
}

void output_matrix(const orc_header* h, int exposure, float* m) {  // demosaic.rs:138-153
    double gain = double(h->gain);
    if (exposure == 0) gain = gain * 10.0 / 9.0;
    for (int i = 0; i < 9; i++) {
        int row = i / 3, col = i % 3;
        double v = XYZ_TO_REC2020[row][0] * double(h->color_matrix[0 * 3 + col]) +
                   XYZ_TO_REC2020[row][1] * double(h->color_matrix[1 * 3 + col]) +
                   XYZ_TO_REC2020[row][2] * double(h->color_matrix[2 * 3 + col]);
        m[i] = float(v * gain);
    }
}

const size_t BAND = 32;  // demosaic.rs:402

}  // namespace

// ===========================================================================
// C ABI
extern "C" {

void orc_codeword(uint32_t p, uint16_t cb, uint32_t* value, uint32_t* len) {
    codeword(p, cb, *value, *len);
}

int orc_read_symbols(const uint8_t* data, size_t len, size_t align, const uint16_t* cbs, size_t n,
                     uint32_t* out) {
    BitReader r(data, len, align);
    for (size_t i = 0; i < n; i++) {
        if (r.top() == 0) return int(i);
        uint32_t v, l;
        codeword(r.top(), cbs[i], v, l);
        r.consume(l);
        out[i] = v;
    }
    return int(n);
}

void orc_decode_component_reduced(const uint8_t* data, size_t len, size_t align,
                                  uint8_t log2_blocks, uint8_t log2_coefs, int16_t* coefs) {
    decode_component_reduced(data, len, align, log2_blocks, log2_coefs, coefs);
}

int16_t orc_dequantize(int16_t coef, int16_t q) { return dequantize(coef, q); }
void orc_apple_block(const int16_t* c, const int16_t* q, uint16_t* o) { apple_block(c, q, o); }
void orc_ffmpeg_block(const int16_t* c, const int16_t* q, uint16_t* o) { ffmpeg_block(c, q, o); }
void orc_apple_block_4x4(const int16_t* c, const int16_t* q, uint16_t* o) { apple_block_4x4(c, q, o); }
void orc_apple_block_2x2(const int16_t* c, const int16_t* q, uint16_t* o) { apple_block_2x2(c, q, o); }
uint16_t orc_output_code(float v) { return output_code(v); }
uint16_t orc_code_value(int32_t c) { return code_value(c); }

void orc_transform_blocks(int idct, const int16_t* coefs, const int16_t* q, uint16_t* out,
                          size_t n) {
    parallel_for((n + 4095) / 4096, 0, [&](size_t chunk) {
        size_t end = std::min(n, (chunk + 1) * 4096);
        for (size_t i = chunk * 4096; i < end; i++) {
            if (idct == 0)
                apple_block(coefs + 64 * i, q + 64 * i, out + 64 * i);
            else
                ffmpeg_block(coefs + 64 * i, q + 64 * i, out + 64 * i);
        }
    });
}

uint16_t orc_curve_linearize(const uint16_t* curve, uint16_t code) {
    return curve_linearize(curve, code);
}

int orc_header_len(const uint8_t* pkt, size_t len, size_t* out, orc_error* err) {
    return header_len(pkt, len, out, err);
}

int orc_parse_header(const uint8_t* pkt, size_t len, orc_header* out, orc_error* err) {
    return parse_header(pkt, len, out, err);
}

int orc_parse_frame(const uint8_t* pkt, size_t len, orc_header* hdr, size_t* ntiles,
                    size_t* tiles_per_row, size_t* tile_rows, uint64_t* tile_off,
                    uint64_t* tile_len, uint8_t* max_qscale, orc_error* err) {
    Parsed p;
    int rc = parse_frame(pkt, len, p, err);
    if (rc) return rc;
    if (hdr) *hdr = p.header;
    if (ntiles) *ntiles = p.off.size();
    if (tiles_per_row) *tiles_per_row = p.tiles_per_row;
    if (tile_rows) *tile_rows = p.rows;
    for (size_t i = 0; i < p.off.size(); i++) {
        if (tile_off) tile_off[i] = p.off[i];
        if (tile_len) tile_len[i] = p.len[i];
    }
    if (max_qscale) *max_qscale = p.max_qscale;
    return ORC_OK;
}

int orc_tile_parse(const uint8_t* data, size_t len, size_t index, uint8_t* qscale,
                   uint64_t* stream_off, uint64_t* stream_len) {
    (void)index;
    Tile t;
    if (!tile_parse(data, len, t)) return ORC_ERR_BAD_TILE_HEADER;
    *qscale = t.qscale;
    for (int s = 0; s < 4; s++) {
        stream_off[s] = t.soff[s];
        stream_len[s] = t.slen[s];
    }
    return ORC_OK;
}

size_t orc_grid_row(size_t width, size_t height, uint8_t alignment, size_t* x,
                    uint8_t* log2_blocks) {
    Grid g(width, height, alignment);
    auto row = g.row();
    for (size_t i = 0; i < row.size(); i++) {
        if (x) x[i] = row[i].x;
        if (log2_blocks) log2_blocks[i] = uint8_t(row[i].log2);
    }
    return row.size();
}

int orc_decode_frame(const uint8_t* pkt, size_t len, int idct, uint16_t* samples,
                     size_t samples_len, uint64_t* skipped, size_t skipped_cap,
                     size_t* n_skipped, uint8_t* max_qscale, orc_header* hdr, int threads,
                     orc_error* err) {
    Parsed p;
    int rc = parse_frame(pkt, len, p, err);
    if (rc) return rc;
    const orc_header& h = p.header;
    const size_t stride = (size_t(h.width) + 15) & ~size_t(15);
    const size_t coded_h = (size_t(h.height) + 15) & ~size_t(15);
    if (samples_len != stride * coded_h) {
        set_err(err, ORC_ERR_BUFFER);
        return ORC_ERR_BUFFER;
    }
    std::memset(samples, 0, sizeof(uint16_t) * samples_len);  // decoder.rs:230
    Grid grid(h.width, h.height, h.alignment);
    const auto row_geo = grid.row();
    const size_t per_row = p.tiles_per_row;
    int ph[4][2];
    stream_phases(h.bayer_pattern, ph);
    std::vector<std::vector<uint64_t>> skip(p.rows);
    parallel_for(p.rows, threads, [&](size_t tr) {  // decoder.rs:238-254
        uint16_t* rows = samples + tr * stride * 16;
        for (size_t i = 0; i < per_row; i++) {
            size_t idx = tr * per_row + i;
            Tile t;
            if (tile_parse(pkt + p.off[idx], p.len[idx], t))
                decode_tile(pkt, p.off[idx], t, row_geo[i], h.quant_matrix, ph, idct, rows, stride);
            else
                skip[tr].push_back(idx);
        }
    });
    size_t n = 0;
    for (auto& v : skip)
        for (auto i : v) {
            if (n < skipped_cap && skipped) skipped[n] = i;
            n++;
        }
    if (n_skipped) *n_skipped = n;
    if (max_qscale) *max_qscale = p.max_qscale;
    if (hdr) *hdr = h;
    return ORC_OK;
}

int orc_decode_frame_reduced(const uint8_t* pkt, size_t len, int log2_factor, int greens,
                             uint16_t* samples, size_t samples_len, uint64_t* skipped,
                             size_t skipped_cap, size_t* n_skipped, uint8_t* max_qscale,
                             orc_header* hdr, int threads, orc_error* err) {
    // reduced.rs:147-201 and TileContext::decode reduced.rs:217-273
    Parsed p;
    int rc = parse_frame(pkt, len, p, err);
    if (rc) return rc;
    const orc_header& h = p.header;
    const uint32_t shift = uint32_t(log2_factor);
    const uint32_t log2_coefs = shift == 1 ? 6 : shift == 2 ? 4 : 2;
    const size_t coded_w = (size_t(h.width) + 15) & ~size_t(15);
    const size_t coded_h = (size_t(h.height) + 15) & ~size_t(15);
    const size_t stride = coded_w >> shift;
    const size_t rows_per_tile = 16 >> shift;
    const size_t side = 16 >> shift;
    if (samples_len != 3 * stride * (coded_h >> shift)) {
        set_err(err, ORC_ERR_BUFFER);
        return ORC_ERR_BUFFER;
    }
    std::memset(samples, 0, sizeof(uint16_t) * samples_len);
    const auto lut = curve_lut(h.curve);
    Grid grid(h.width, h.height, h.alignment);
    const auto row_geo = grid.row();
    const size_t per_row = p.tiles_per_row;
    std::vector<std::vector<uint64_t>> skip(p.rows);
    parallel_for(p.rows, threads, [&](size_t tr) {
        uint16_t* rows = samples + tr * 3 * stride * rows_per_tile;
        for (size_t ti = 0; ti < per_row; ti++) {
            size_t idx = tr * per_row + ti;
            Tile t;
            if (!tile_parse(pkt + p.off[idx], p.len[idx], t)) {
                skip[tr].push_back(idx);
                continue;
            }
            const Geometry& g = row_geo[ti];
            int16_t q[64];
            for (int i = 0; i < 64; i++) q[i] = int16_t(uint16_t(h.quant_matrix[i]) * uint16_t(t.qscale));
            const size_t per_block = size_t(1) << log2_coefs;
            const size_t blocks = size_t(1) << g.log2;
            const size_t x0 = g.x >> shift;
            int16_t coefs[64 * 16];
            const int plan[4][3] = {{0, 3, 0}, {1, 0, 0}, {1, 1, 1}, {2, 2, 0}};
            for (int k = 0; k < 4; k++) {
                int channel = plan[k][0], stream = plan[k][1], average = plan[k][2];
                if (average && !greens) continue;
                size_t off = p.off[idx] + t.soff[stream];
                decode_component_reduced(pkt + off, t.slen[stream], off & 3, g.log2, log2_coefs, coefs);
                for (size_t b = 0; b < blocks; b++) {
                    uint16_t values[64];
                    const int16_t* blk = coefs + per_block * b;
                    if (shift == 1)
                        apple_block(blk, q, values);
                    else if (shift == 2)
                        apple_block_4x4(blk, q, values);
                    else
                        apple_block_2x2(blk, q, values);
                    size_t bx = x0 + b * side;
                    for (size_t i = 0; i < side; i++) {
                        uint16_t* d = rows + 3 * (i * stride + bx) + channel;
                        for (size_t j = 0; j < side; j++) {
                            uint16_t v = values[i * side + j];
                            if (average) {
                                uint32_t sum = uint32_t(d[3 * j]) + uint32_t(lut[v]);
                                d[3 * j] = uint16_t((sum + 1) / 2);
                            } else {
                                d[3 * j] = lut[v];
                            }
                        }
                    }
                }
            }
        }
    });
    size_t n = 0;
    for (auto& v : skip)
        for (auto i : v) {
            if (n < skipped_cap && skipped) skipped[n] = i;
            n++;
        }
    if (n_skipped) *n_skipped = n;
    if (max_qscale) *max_qscale = p.max_qscale;
    if (hdr) *hdr = h;
    return ORC_OK;
}

int orc_linearize(const orc_header* hdr, const uint16_t* samples, uint16_t* out, size_t out_len,
                  int threads) {
    // decoder.rs:197-216
    const size_t w = hdr->width, h = hdr->height;
    const size_t stride = (w + 15) & ~size_t(15);
    if (out_len != w * h) return ORC_ERR_BUFFER;
    if (w == 0) return ORC_OK;
    const auto lut = curve_lut(hdr->curve);
    parallel_for(h, threads, [&](size_t y) {
        for (size_t x = 0; x < w; x++) out[y * w + x] = lut[samples[y * stride + x]];
    });
    return ORC_OK;
}

void orc_params_with_white_balance(const orc_header* hdr, uint32_t quantizer, float red,
                                   float blue, orc_params* out) {
    // demosaic.rs:86-106
    uint32_t range = uint16_t(hdr->white_level - 256);
    double q = double(quantizer);
    double base = q * q * 5.0 + 64.0 / 3.0;
    double range2 = double(range) * double(range);
    float rangef = float(range);
    auto inverse = [](float g) { return g == 0.0f ? 1.0f : 1.0f / g; };
    out->cfa_phase = hdr->bayer_pattern;
    out->black = 256;
    out->one_over_range = 1.0f / rangef;
    out->noise[0] = float(base / 150994944.0);
    out->noise[1] = float(base / (range2 * 256.0));
    out->noise[2] = float(64.0 / 3.0 / range2);
    out->clip[0] = inverse(red);
    out->clip[1] = inverse(blue);
    out->black_over_range = 256.0f / rangef;
    out->wb[0] = red;
    out->wb[1] = blue;
}

void orc_output_matrix(const orc_header* hdr, int exposure, float* m9) {
    output_matrix(hdr, exposure, m9);
}

int orc_develop(const orc_header* hdr, const uint16_t* samples, const orc_params* params,
                int stage, int planar, float* r_out, float* g_out, float* b_out, size_t out_len,
                int threads) {
    // develop_into / develop_planar_into, demosaic.rs:223-261, Conversion demosaic.rs:286-398
    const size_t w = hdr->width, h = hdr->height;
    const size_t stride = (w + 15) & ~size_t(15);
    if (planar ? out_len != w * h : out_len != 3 * w * h) return ORC_ERR_BUFFER;
    orc_params p = *params;
    if (stage == 0) {
        p.wb[0] = p.wb[1] = 1.0f;
        p.clip[0] = p.clip[1] = 1.0f;
    }
    float m[9];
    const bool has_matrix = stage == 2;
    if (has_matrix) output_matrix(hdr, 0, m);
    const auto clut = curve_lut(hdr->curve);
    std::vector<float> lut(65536);
    for (size_t i = 0; i < 65536; i++) lut[i] = p.one_over_range * float(int32_t(clut[i]) - p.black);
    const size_t nbands = (h + BAND - 1) / BAND;
    parallel_for(nbands, threads, [&](size_t index) {  // band, demosaic.rs:356-398
        size_t y0 = index * BAND;
        size_t y1 = std::min(y0 + BAND, h);
        size_t g0 = y0 > 0 ? y0 - 1 : 0, g1 = std::min(y1 + 1, h);
        size_t n0 = g0 >= 2 ? g0 - 2 : 0, n1 = std::min(g1 + 2, h);
        std::vector<float> norm((n1 - n0) * w);
        for (size_t y = n0; y < n1; y++)
            for (size_t x = 0; x < w; x++) norm[(y - n0) * w + x] = lut[samples[y * stride + x]];
        std::vector<float> green((g1 - g0) * w * 2);
        for (size_t y = g0; y < g1; y++) {
            const float* rows[5];
            for (int k = 0; k < 5; k++) {
                long yy = std::clamp(long(y) + k - 2, 0L, long(h) - 1);
                rows[k] = norm.data() + (size_t(yy) - n0) * w;
            }
            green_row(rows, y, h, w, p, green.data() + (y - g0) * w * 2);
        }
        auto grow = [&](size_t yy) { return green.data() + (yy - g0) * w * 2; };
        for (size_t y = y0; y < y1; y++) {
            size_t ym, yp;
            mirrored(y, h, ym, yp);
            chroma_row(grow(ym), grow(y), grow(yp), w, y, p,
                       [&](size_t x, float r, float g, float b) {
                           if (has_matrix) matrix_px(r, g, b, m);
                           if (planar) {
                               r_out[y * w + x] = r;
                               g_out[y * w + x] = g;
                               b_out[y * w + x] = b;
                           } else {
                               float* o = r_out + 3 * (y * w + x);
                               o[0] = r;
                               o[1] = g;
                               o[2] = b;
                           }
                       });
        }
    });
    return ORC_OK;
}

void orc_green_pass(const uint16_t* linear, size_t w, size_t h, const orc_params* params,
                    float* out2) {
    // demosaic.rs:453-476
    const orc_params& p = *params;
    std::vector<float> norm(w * h);
    for (size_t i = 0; i < w * h; i++) norm[i] = p.one_over_range * float(int32_t(linear[i]) - p.black);
    for (size_t y = 0; y < h; y++) {
        const float* rows[5];
        for (int k = 0; k < 5; k++) {
            long yy = std::clamp(long(y) + k - 2, 0L, long(h) - 1);
            rows[k] = norm.data() + size_t(yy) * w;
        }
        green_row(rows, y, h, w, p, out2 + y * w * 2);
    }
}

void orc_chroma_pass(const float* green2, size_t w, size_t h, const orc_params* params,
                     float* out3) {
    // demosaic.rs:608-617
    for (size_t y = 0; y < h; y++) {
        size_t ym, yp;
        mirrored(y, h, ym, yp);
        chroma_row(green2 + ym * w * 2, green2 + y * w * 2, green2 + yp * w * 2, w, y, *params,
                   [&](size_t x, float r, float g, float b) {
                       out3[3 * (y * w + x)] = r;
                       out3[3 * (y * w + x) + 1] = g;
                       out3[3 * (y * w + x) + 2] = b;
                   });
    }
}

void orc_apply_matrix(const float* rgb, size_t n_px, const float* m9, float* out) {
    // demosaic.rs:692-707
    for (size_t i = 0; i < n_px; i++) {
        float r = rgb[3 * i], g = rgb[3 * i + 1], b = rgb[3 * i + 2];
        matrix_px(r, g, b, m9);
        out[3 * i] = r;
        out[3 * i + 1] = g;
        out[3 * i + 2] = b;
    }
}

}  // extern "C"
