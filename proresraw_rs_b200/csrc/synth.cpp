// synth.cpp -- synthetic ProRes RAW input (libprr_synth.so). See include/prr_synth.h.
//
// Part 1 restates the crate's test support (src/synth.rs, src/idct.rs testgen)
// so that parity corpora are built exactly as the crate's own tests build
// them. Part 2 is new: a mosaic generator and an encoder, because the crate
// has no encoder and the benchmark frames must be real encoded mosaics.

#include "../../include/prr_synth.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <functional>
#include <thread>
#include <vector>

namespace {

void parallel_for(size_t n, int threads, const std::function<void(size_t)>& f) {
    size_t t = threads > 0 ? size_t(threads) : std::max(1u, std::thread::hardware_concurrency());
    t = std::min(t, n);
    if (t <= 1) {
        for (size_t i = 0; i < n; i++) f(i);
        return;
    }
    std::atomic<size_t> next{0};
    std::vector<std::thread> pool;
    for (size_t k = 0; k < t; k++)
        pool.emplace_back([&] {
            for (size_t i = next.fetch_add(1); i < n; i = next.fetch_add(1)) f(i);
        });
    for (auto& th : pool) th.join();
}

void put_be16(std::vector<uint8_t>& v, uint16_t x) {
    v.push_back(uint8_t(x >> 8));
    v.push_back(uint8_t(x));
}
void set_be16(uint8_t* p, uint16_t x) {
    p[0] = uint8_t(x >> 8);
    p[1] = uint8_t(x);
}
void set_bef32(uint8_t* p, float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    p[0] = uint8_t(u >> 24);
    p[1] = uint8_t(u >> 16);
    p[2] = uint8_t(u >> 8);
    p[3] = uint8_t(u);
}
uint16_t be16(const uint8_t* p) { return uint16_t(p[0] << 8 | p[1]); }

// Tile grid, bitstream description section 4 (src/tile.rs:46-107).
struct Geo {
    size_t x;
    uint32_t log2;
};
std::vector<Geo> grid_row(size_t width, uint32_t alignment) {
    std::vector<Geo> out;
    size_t column = 0, remaining = (width + 15) / 16;
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

// Stream s lands on Bayer phase (row, col) (src/header.rs:64-82).
void stream_phases(uint8_t pattern, int ph[4][2]) {
    int r = (pattern == 2 || pattern == 3) ? 1 : 0;
    int c = (pattern == 1 || pattern == 3) ? 1 : 0;
    ph[0][0] = 1 - r; ph[0][1] = c;
    ph[1][0] = r;     ph[1][1] = 1 - c;
    ph[2][0] = 1 - r; ph[2][1] = 1 - c;
    ph[3][0] = r;     ph[3][1] = c;
}

struct Rng {  // src/synth.rs:9-29
    uint64_t s;
    uint32_t next_u32() {
        s ^= s >> 12;
        s ^= s << 25;
        s ^= s >> 27;
        return uint32_t((s * 0x2545F4914F6CDD1DULL) >> 32);
    }
    uint32_t below(uint32_t b) { return next_u32() % b; }
};

// Header body + packet assembly, src/synth.rs:99-152.
std::vector<uint8_t> frame_packet(const prs_spec& spec, const std::vector<std::vector<uint8_t>>& tiles) {
    uint16_t flags = uint16_t(spec.alignment) << 1;
    std::vector<uint8_t> body(70, 0);
    body[1] = spec.version;
    std::memcpy(&body[2], spec.vendor, 4);
    set_be16(&body[6], spec.width);
    set_be16(&body[8], spec.height);
    std::memcpy(&body[10], spec.crop, 4);
    set_be16(&body[14], spec.pattern);
    set_be16(&body[16], uint16_t(spec.white_level - 256));
    set_bef32(&body[18], spec.wb[0]);
    set_bef32(&body[22], spec.wb[1]);
    for (int i = 0; i < 9; i++) set_bef32(&body[26 + 4 * i], spec.color_matrix[i]);
    set_bef32(&body[62], spec.gain);
    set_be16(&body[66], spec.wb_cct);
    if (spec.has_quant_matrix) {
        flags |= 1;
        body.insert(body.end(), spec.quant_matrix, spec.quant_matrix + 64);
    }
    if (spec.has_curve) {
        flags |= 1 << 4;
        for (int i = 0; i < 8; i++) put_be16(body, spec.curve[i]);
    }
    set_be16(&body[68], flags);
    std::vector<uint8_t> pkt;
    size_t total = 10 + body.size() + 2 * tiles.size();
    for (auto& t : tiles) total += t.size();
    pkt.reserve(total);
    pkt.resize(4, 0);
    pkt.insert(pkt.end(), {'p', 'r', 'r', 'f'});
    put_be16(pkt, uint16_t(body.size() + 2));
    pkt.insert(pkt.end(), body.begin(), body.end());
    for (auto& t : tiles) put_be16(pkt, uint16_t(t.size()));
    for (auto& t : tiles) pkt.insert(pkt.end(), t.begin(), t.end());
    uint32_t len = uint32_t(pkt.size());
    pkt[0] = uint8_t(len >> 24);
    pkt[1] = uint8_t(len >> 16);
    pkt[2] = uint8_t(len >> 8);
    pkt[3] = uint8_t(len);
    return pkt;
}

std::vector<uint8_t> make_tile(uint8_t qscale, const std::vector<uint8_t>* streams[4]) {  // synth.rs:175-184
    std::vector<uint8_t> t = {uint8_t(8 << 3), qscale};
    for (int s = 0; s < 3; s++) put_be16(t, uint16_t(streams[s]->size()));
    for (int s = 0; s < 4; s++) t.insert(t.end(), streams[s]->begin(), streams[s]->end());
    return t;
}

std::vector<uint8_t> random_tile(size_t blocks, bool valid, Rng& rng) {  // synth.rs:158-170
    uint32_t floor = valid ? 1 : 0;
    uint8_t qscale = uint8_t(floor + rng.below(256 - floor));
    uint32_t sizes[4];
    for (int s = 0; s < 4; s++) sizes[s] = floor + rng.below(uint32_t(48 * blocks + 1) - floor);
    std::vector<uint8_t> streams[4];
    for (int s = 0; s < 4; s++) {
        streams[s].resize(sizes[s]);
        for (uint32_t i = 0; i < sizes[s]; i++) {
            uint32_t a = rng.next_u32();
            uint32_t b = rng.next_u32();
            streams[s][i] = uint8_t(a & b);
        }
    }
    const std::vector<uint8_t>* ptrs[4] = {&streams[0], &streams[1], &streams[2], &streams[3]};
    return make_tile(qscale, ptrs);
}

// ---------------------------------------------------------------------------
// Codeword writer (bitstream description section 6.1; src/bits.rs:136-186).
struct BitWriter {
    std::vector<uint8_t> bytes;
    uint64_t acc = 0;
    int nacc = 0;
    void put(uint32_t value, uint32_t n) {
        // n <= 32
        if (n == 0) return;
        acc = (acc << n) | (uint64_t(value) & ((n == 32) ? 0xFFFFFFFFull : ((1ull << n) - 1)));
        nacc += int(n);
        while (nacc >= 8) {
            bytes.push_back(uint8_t(acc >> (nacc - 8)));
            nacc -= 8;
        }
    }
    void put_zeros(uint32_t n) {
        while (n > 32) {
            put(0, 32);
            n -= 32;
        }
        put(0, n);
    }
    std::vector<uint8_t> finish() {
        if (nacc > 0) {
            bytes.push_back(uint8_t(acc << (8 - nacc)));
            nacc = 0;
        }
        return std::move(bytes);
    }
};

inline uint32_t cw_len(uint16_t cb, uint32_t v) {
    uint32_t s = cb >> 8, e = (cb >> 4) & 15, r = cb & 15;
    uint32_t q = v >> r;
    if (q <= s) return q + 1 + r;
    uint32_t m = v - ((s + 1) << r) + (1u << e);
    uint32_t bits = 32 - uint32_t(__builtin_clz(m));
    return s + 1 + (bits - 1 - e) + bits;
}

inline uint32_t put_symbol(BitWriter& w, uint16_t cb, uint32_t v) {
    uint32_t s = cb >> 8, e = (cb >> 4) & 15, r = cb & 15;
    uint32_t q = v >> r;
    if (q <= s) {
        w.put_zeros(q);
        w.put(1, 1);
        w.put(v & ((1u << r) - 1), r);
        return q + 1 + r;
    }
    uint32_t m = v - ((s + 1) << r) + (1u << e);
    uint32_t bits = 32 - uint32_t(__builtin_clz(m));
    uint32_t zeros = s + 1 + (bits - 1 - e);
    w.put_zeros(zeros);
    w.put(m, bits);
    return zeros + bits;
}

// Codebook tables, bitstream description section 6.3-6.5.
const uint16_t FIRST_DC = 0x2BC, DC_RESET = 0x064, AC_INITIAL = 0x031, RN_INITIAL = 0x000,
               LN_INITIAL = 0x042;
const uint16_t DC_CB[13] = {0x010, 0x021, 0x032, 0x033, 0x033, 0x033, 0x044,
                            0x044, 0x044, 0x044, 0x044, 0x044, 0x076};
const uint16_t RN_CB[28] = {0x200, 0x100, 0x000, 0x000, 0x211, 0x211, 0x111, 0x111, 0x011, 0x011,
                            0x021, 0x021, 0x222, 0x022, 0x022, 0x022, 0x022, 0x022, 0x022, 0x022,
                            0x022, 0x022, 0x022, 0x022, 0x022, 0x032, 0x032, 0x044};
const uint16_t LN_CB[15] = {0x100, 0x111, 0x222, 0x222, 0x122, 0x122, 0x433, 0x433,
                            0x233, 0x233, 0x233, 0x233, 0x233, 0x233, 0x033};
uint16_t ac_cb(uint32_t symbol) {
    static const int counts[10] = {1, 1, 2, 3, 3, 8, 2, 22, 52, 1};
    static const uint16_t vals[10] = {0x000, 0x211, 0x111, 0x222, 0x122,
                                      0x233, 0x133, 0x244, 0x355, 0x166};
    uint32_t i = std::min<uint32_t>(symbol, 94);
    for (int r = 0; r < 10; r++) {
        if (i < uint32_t(counts[r])) return vals[r];
        i -= counts[r];
    }
    return 0x166;
}
const uint8_t SCAN[64] = {0,  8,  1,  9,  16, 24, 17, 25, 2,  10, 3,  11, 18, 26, 19, 27,
                          32, 40, 33, 34, 41, 48, 56, 49, 42, 35, 43, 50, 57, 58, 51, 59,
                          4,  12, 5,  6,  13, 20, 28, 21, 14, 7,  15, 22, 29, 36, 44, 37,
                          30, 23, 31, 38, 45, 52, 60, 53, 46, 39, 47, 54, 61, 62, 55, 63};

// Entropy-code one component: `coefs` holds `blocks` raster-order blocks.
// Written against the decoder's rules (section 6.2-6.4); every codeword is
// kept within 32 bits (31 for levels, whose sign bit follows) by clamping
// the value toward zero, which only makes the encoder lossier.
std::vector<uint8_t> encode_component(const int16_t* coefs, uint32_t log2_blocks) {
    const uint32_t blocks = 1u << log2_blocks;
    const uint32_t codes = 64 * blocks;
    auto at = [&](uint32_t n) -> int32_t {
        return coefs[64 * (n & (blocks - 1)) + SCAN[n >> log2_blocks]];
    };
    BitWriter w;
    // DC: folded first value, then deltas with a running sign.
    int32_t dc = at(0);
    uint32_t folded = dc >= 0 ? uint32_t(2 * dc) : uint32_t(-2 * dc - 1);
    put_symbol(w, FIRST_DC, folded);
    uint16_t dc_cb = DC_RESET;
    uint32_t sign = 0;
    for (uint32_t b = 1; b < blocks; b++) {
        int32_t want = at(b) - dc;
        uint32_t sym = 0, mag = 0;
        for (;;) {
            mag = uint32_t(want < 0 ? -want : want);
            if (want == 0) {
                sym = 0;
            } else if (want > 0) {
                sym = sign ? 2 * mag - 1 : 2 * mag;
            } else {
                sym = (1 ^ sign) ? 2 * mag - 1 : 2 * mag;
            }
            if (cw_len(dc_cb, sym) <= 32) break;
            want = want > 0 ? want - 1 : want + 1;
        }
        put_symbol(w, dc_cb, sym);
        uint32_t odd = sym & 1;
        sign ^= odd;
        uint32_t magnitude = (odd + sym) >> 1;
        int32_t delta = sign ? -int32_t(magnitude) : int32_t(magnitude);
        dc_cb = DC_CB[std::min<uint32_t>(magnitude, 12)];
        sign = delta < 0 ? 1 : 0;
        dc += delta;
    }
    // AC: runs of non-zero levels and runs of zeros.
    int64_t last = -1;
    for (uint32_t n = codes; n-- > blocks;) {
        if (at(n) != 0) {
            last = n;
            break;
        }
    }
    uint16_t acb = AC_INITIAL, rnb = RN_INITIAL, lnb = LN_INITIAL;
    auto level = [&](int32_t v) -> uint32_t {
        uint32_t mag = uint32_t(v < 0 ? -v : v);
        uint32_t sym = mag - 1;
        while (sym > 0 && cw_len(acb, sym) > 31) sym--;
        put_symbol(w, acb, sym);
        w.put(v < 0 ? 1 : 0, 1);
        acb = ac_cb(sym);
        return sym;
    };
    uint32_t n = blocks;
    if (last >= int64_t(blocks)) {
        for (;;) {
            uint32_t L = 0;
            while (n + L < codes && at(n + L) != 0) L++;
            put_symbol(w, lnb, L);
            for (uint32_t k = 0; k < L; k++) level(at(n + k));
            n += L;
            if (n == codes || int64_t(n) > last) break;
            uint32_t z = 0;
            while (at(n + z) == 0) z++;
            put_symbol(w, rnb, z - 1);
            rnb = RN_CB[std::min<uint32_t>(z - 1, 27)];
            n += z;
            uint32_t sym = level(at(n));
            lnb = LN_CB[std::min<uint32_t>(sym, 14)];
            n += 1;
            if (n >= codes || int64_t(n) > last) break;
        }
    }
    return w.finish();
}

// Forward 8x8 DCT matched to the decoder's scaling: the inverse transforms
// give out[y][x] = 2 * sum_{v,u} c_u c_v C[v][u] cos((2x+1)u pi/16) cos((2y+1)v pi/16)
// (+32768), so C[v][u] = (1/32) c_u c_v sum f cos cos, with c_0 = 1/sqrt(2).
struct Dct {
    double k[8][8];  // k[u][x] = c_u cos((2x+1) u pi / 16)
    Dct() {
        for (int u = 0; u < 8; u++)
            for (int x = 0; x < 8; x++)
                k[u][x] = (u == 0 ? std::sqrt(0.5) : 1.0) * std::cos((2 * x + 1) * u * M_PI / 16.0);
    }
    void forward(const double f[8][8], double C[8][8]) const {
        double t[8][8];
        for (int y = 0; y < 8; y++)
            for (int u = 0; u < 8; u++) {
                double s = 0;
                for (int x = 0; x < 8; x++) s += f[y][x] * k[u][x];
                t[y][u] = s;
            }
        for (int v = 0; v < 8; v++)
            for (int u = 0; u < 8; u++) {
                double s = 0;
                for (int y = 0; y < 8; y++) s += t[y][u] * k[v][y];
                C[v][u] = s / 32.0;
            }
    }
};
const Dct DCT;

uint16_t curve_linearize(const uint16_t* curve, uint32_t code) {  // section 8
    uint32_t seg = code >> 13, frac = code & 0x1FFF;
    uint32_t c0 = curve[seg];
    uint32_t c1 = seg < 7 ? curve[seg + 1] : 65536u;
    uint32_t delta = (c1 - c0) & 0xFFFF;
    return uint16_t(std::min<uint32_t>((c0 * 8192 + delta * frac + 4096) >> 13, 65535));
}

}  // namespace

extern "C" {

uint64_t prs_rng_new(uint64_t seed) { return (seed * 0x9E3779B97F4A7C15ULL) | 1; }
uint32_t prs_rng_next_u32(uint64_t* state) {
    Rng r{*state};
    uint32_t v = r.next_u32();
    *state = r.s;
    return v;
}
uint32_t prs_rng_below(uint64_t* state, uint32_t bound) {
    return prs_rng_next_u32(state) % bound;
}

void prs_spec_new(uint16_t width, uint16_t height, uint8_t pattern, prs_spec* s) {
    std::memset(s, 0, sizeof(*s));
    s->width = width;
    s->height = height;
    s->alignment = 3;
    s->pattern = pattern;
    std::memcpy(s->vendor, "test", 4);
    s->white_level = 0xFDFF + 256;
    s->wb[0] = s->wb[1] = 1.0f;
    s->color_matrix[0] = s->color_matrix[4] = s->color_matrix[8] = 1.0f;
    s->gain = 1.0f;
    s->wb_cct = 5600;
    s->valid_tiles = 0;
    s->version = 1;
}

size_t prs_specs(uint64_t* state, prs_spec* out, size_t cap) {
    Rng rng{*state};
    size_t n = 0;
    for (uint8_t alignment = 0; alignment <= 4; alignment++) {
        for (uint8_t i = 0; i < 4; i++) {
            uint16_t width = uint16_t(2 * (1 + rng.below(300)));
            uint16_t height = uint16_t(2 * (1 + rng.below(40)));
            prs_spec s;
            prs_spec_new(width, height, i, &s);
            s.alignment = alignment;
            if (i == 1) {
                s.has_quant_matrix = 1;
                std::fill(s.quant_matrix, s.quant_matrix + 64, 63);
            } else if (i >= 2) {
                s.has_quant_matrix = 1;
                for (int k = 0; k < 64; k++) s.quant_matrix[k] = uint8_t(1 + rng.below(63));
            }
            if (i % 2 == 1) {
                uint16_t c[8];
                for (int k = 0; k < 8; k++) c[k] = uint16_t(rng.below(65536 - 8));
                std::sort(c, c + 8);
                s.has_curve = 1;
                for (int k = 0; k < 8; k++) s.curve[k] = uint16_t(c[k] + k);
            }
            if (n < cap) out[n] = s;
            n++;
        }
    }
    *state = rng.s;
    return n;
}

size_t prs_random_frame(const prs_spec* spec, uint64_t* state, uint8_t* out, size_t cap) {
    Rng rng{*state};
    auto row = grid_row(spec->width, spec->alignment);
    size_t rows = (size_t(spec->height) + 15) / 16;
    std::vector<std::vector<uint8_t>> tiles;
    tiles.reserve(row.size() * rows);
    for (size_t r = 0; r < rows; r++)
        for (auto& g : row) tiles.push_back(random_tile(size_t(1) << g.log2, spec->valid_tiles != 0, rng));
    auto pkt = frame_packet(*spec, tiles);
    if (cap == 0) return pkt.size();
    if (pkt.size() > cap) return 0;
    std::memcpy(out, pkt.data(), pkt.size());
    *state = rng.s;
    return pkt.size();
}

size_t prs_frame_from_tiles(const prs_spec* spec, const uint8_t* tiles, const uint32_t* tile_lens,
                            size_t ntiles, uint8_t* out, size_t cap) {
    std::vector<std::vector<uint8_t>> t(ntiles);
    size_t off = 0;
    for (size_t i = 0; i < ntiles; i++) {
        t[i].assign(tiles + off, tiles + off + tile_lens[i]);
        off += tile_lens[i];
    }
    auto pkt = frame_packet(*spec, t);
    if (pkt.size() > cap) return pkt.size();
    std::memcpy(out, pkt.data(), pkt.size());
    return pkt.size();
}

size_t prs_tile(uint8_t qscale, const uint8_t* const streams[4], const uint32_t lens[4], uint8_t* out,
                size_t cap) {
    std::vector<uint8_t> s[4];
    for (int i = 0; i < 4; i++) s[i].assign(streams[i], streams[i] + lens[i]);
    const std::vector<uint8_t>* p[4] = {&s[0], &s[1], &s[2], &s[3]};
    auto t = make_tile(qscale, p);
    if (t.size() > cap) return t.size();
    std::memcpy(out, t.data(), t.size());
    return t.size();
}

size_t prs_bitwrite(const prs_bitop* ops, size_t n, uint8_t* out, size_t cap) {
    BitWriter w;
    for (size_t i = 0; i < n; i++) {
        if (ops[i].kind == 0)
            put_symbol(w, uint16_t(ops[i].a), ops[i].b);
        else
            w.put(ops[i].b, ops[i].a);
    }
    auto bytes = w.finish();
    if (bytes.size() > cap) return bytes.size();
    std::memcpy(out, bytes.data(), bytes.size());
    return bytes.size();
}

// testgen::Gen, src/idct.rs:363-442.
uint64_t prs_gen_new(uint64_t seed) { return seed; }

static inline uint64_t gen_next(uint64_t& s) {
    s += 0x9e3779b97f4a7c15ULL;
    uint64_t z = s;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

void prs_gen_blocks(uint64_t* state, uint64_t first, size_t n, int16_t* coefs, int16_t* q) {
    uint64_t s = *state;
    auto below = [&](uint64_t m) { return gen_next(s) % m; };
    auto sgn = [&](int32_t m) { return int16_t(int32_t(below(uint64_t(2 * m + 1))) - m); };
    auto qq = [&](uint64_t qmat, uint64_t qscale, int16_t* out) {
        uint64_t sc = 1 + below(qscale);
        for (int k = 0; k < 64; k++) out[k] = int16_t((1 + below(qmat)) * sc);
    };
    for (size_t bi = 0; bi < n; bi++) {
        int16_t* c = coefs + 64 * bi;
        int16_t* qo = q + 64 * bi;
        std::memset(c, 0, 128);
        switch ((first + bi) % 6) {
            case 0:
                qq(63, 255, qo);
                c[0] = int16_t(gen_next(s));
                break;
            case 1: {
                qq(63, 255, qo);
                c[0] = sgn(2047);
                uint64_t cnt = 1 + below(9);
                for (uint64_t i = 0; i < cnt; i++) {
                    size_t k = size_t(below(64));
                    c[k] = sgn(2047);
                }
                break;
            }
            case 2:
                qq(16, 8, qo);
                for (int k = 0; k < 64; k++) c[k] = sgn(255);
                break;
            case 3:
                qq(8, 4, qo);
                for (int k = 0; k < 64; k++) {
                    int32_t m = 4096 >> std::min((k / 8 + k % 8) / 2, 12);
                    c[k] = sgn(m);
                }
                break;
            case 4:
                qq(63, 255, qo);
                for (int k = 0; k < 64; k++) c[k] = int16_t(gen_next(s));
                break;
            default:
                for (int k = 0; k < 64; k++) qo[k] = int16_t(gen_next(s));
                for (int k = 0; k < 64; k++) c[k] = int16_t(gen_next(s));
                break;
        }
    }
    *state = s;
}

uint64_t prs_fnv1a_u16(uint64_t h, const uint16_t* v, size_t n) {
    for (size_t i = 0; i < n; i++) {
        h ^= uint64_t(v[i] & 0xFF);
        h *= 0x00000100000001b3ULL;
        h ^= uint64_t(v[i] >> 8);
        h *= 0x00000100000001b3ULL;
    }
    return h;
}

void prs_mosaic(const prs_mosaic_params* p, uint16_t* out, int threads) {
    Rng rng{prs_rng_new(p->seed)};
    struct Wave {
        double amp, kx, ky, phase;
    } waves[3];
    for (auto& wv : waves) {
        double amp = p->amp_lo + (p->amp_hi - p->amp_lo) * (rng.below(1u << 20) / double(1u << 20));
        double wavelength = 256.0 + rng.below(1793);  // 256 .. 2048 sensels
        double angle = 2.0 * M_PI * (rng.below(1u << 20) / double(1u << 20));
        double phase = 2.0 * M_PI * (rng.below(1u << 20) / double(1u << 20));
        wv = {amp, 2.0 * M_PI * std::cos(angle) / wavelength, 2.0 * M_PI * std::sin(angle) / wavelength,
              phase};
    }
    const uint32_t w = p->width, h = p->height;
    const int rr = (p->pattern == 2 || p->pattern == 3) ? 1 : 0;
    const int rc = (p->pattern == 1 || p->pattern == 3) ? 1 : 0;
    const double white = p->white;
    const uint32_t spec_thresh = uint32_t(double(p->specular) * 4294967296.0 > 4294967295.0
                                              ? 4294967295.0
                                              : double(p->specular) * 4294967296.0);
    parallel_for(h, threads, [&](size_t y) {
        Rng r{prs_rng_new(p->seed * 0x100000001B3ULL + y + 1)};
        auto uniform = [&]() { return (r.next_u32() + 0.5) / 4294967296.0; };
        double spare = 0;
        bool have = false;
        auto gauss = [&]() {
            if (have) {
                have = false;
                return spare;
            }
            double u1 = uniform(), u2 = uniform();
            double m = std::sqrt(-2.0 * std::log(u1));
            spare = m * std::sin(2.0 * M_PI * u2);
            have = true;
            return m * std::cos(2.0 * M_PI * u2);
        };
        for (uint32_t x = 0; x < w; x++) {
            double v = 0;
            for (auto& wv : waves) v += wv.amp * 0.5 * (1.0 + std::cos(wv.kx * x + wv.ky * double(y) + wv.phase));
            int color = ((int(y) & 1) == rr && (int(x) & 1) == rc) ? 0
                        : ((int(y) & 1) != rr && (int(x) & 1) != rc) ? 2
                                                                      : 1;
            v = 256.0 + v * p->chan_gain[color];
            if (p->sigma > 0) v += p->sigma * gauss();
            uint32_t sr = r.next_u32();
            if (sr < spec_thresh) v = white;
            v = std::min(std::max(std::round(v), 256.0), white);
            out[size_t(y) * w + x] = uint16_t(v);
        }
    });
}

size_t prs_encode(const prs_encode_params* ep, const uint16_t* mosaic, uint8_t* out, size_t cap,
                  int threads) {
    const prs_spec& spec = ep->spec;
    const size_t w = spec.width, h = spec.height;
    const size_t cw = (w + 15) & ~size_t(15), ch = (h + 15) & ~size_t(15);
    auto row = grid_row(w, spec.alignment);
    const size_t rows = ch / 16;
    const size_t ntiles = row.size() * rows;
    // Linear -> code value through the inverse of the header curve
    // (nearest code whose linearized value matches).
    static const uint16_t DEFAULT_CURVE[8] = {0, 512, 1024, 2048, 4096, 8192, 16384, 32768};
    const uint16_t* curve = spec.has_curve ? spec.curve : DEFAULT_CURVE;
    std::vector<uint16_t> lin(65536);
    for (uint32_t c = 0; c < 65536; c++) lin[c] = curve_linearize(curve, c);
    std::vector<uint16_t> inv(65536);
    {
        uint32_t c = 0;
        for (uint32_t L = 0; L < 65536; L++) {
            while (c < 65535 && lin[c] < L) c++;
            uint32_t best = c;
            if (c > 0 && std::abs(int(lin[c - 1]) - int(L)) <= std::abs(int(lin[c]) - int(L))) best = c - 1;
            inv[L] = uint16_t(best);
        }
    }
    // Code plane padded to the coded size by edge replication.
    std::vector<uint16_t> code(cw * ch);
    parallel_for(ch, threads, [&](size_t y) {
        size_t sy = std::min(y, h - 1);
        for (size_t x = 0; x < cw; x++) code[y * cw + x] = inv[mosaic[sy * w + std::min(x, w - 1)]];
    });
    std::vector<uint8_t> qscales(ntiles);
    {
        Rng r{prs_rng_new(ep->qscale_seed)};
        uint32_t lo = ep->qscale_lo ? ep->qscale_lo : 1, hi = std::max<uint32_t>(ep->qscale_hi, lo);
        for (size_t i = 0; i < ntiles; i++) qscales[i] = uint8_t(lo + r.below(hi - lo + 1));
    }
    uint8_t qmat[64];
    if (spec.has_quant_matrix)
        std::memcpy(qmat, spec.quant_matrix, 64);
    else
        std::fill(qmat, qmat + 64, 1);
    int ph[4][2];
    stream_phases(spec.pattern, ph);
    std::vector<std::vector<uint8_t>> tiles(ntiles);
    std::atomic<bool> too_big{false};
    parallel_for(rows, threads, [&](size_t tr) {
        for (size_t ti = 0; ti < row.size(); ti++) {
            const Geo& g = row[ti];
            size_t idx = tr * row.size() + ti;
            uint8_t qs = qscales[idx];
            size_t blocks = size_t(1) << g.log2;
            std::vector<uint8_t> streams[4];
            std::vector<int16_t> coefs(64 * blocks);
            for (int s = 0; s < 4; s++) {
                for (size_t b = 0; b < blocks; b++) {
                    double f[8][8], C[8][8];
                    for (int i = 0; i < 8; i++)
                        for (int j = 0; j < 8; j++) {
                            size_t yy = tr * 16 + 2 * i + ph[s][0];
                            size_t xx = g.x + 16 * b + 2 * j + ph[s][1];
                            f[i][j] = double(code[yy * cw + xx]) - 32768.0;
                        }
                    DCT.forward(f, C);
                    for (int k = 0; k < 64; k++) {
                        double qv = double(qmat[k]) * qs;
                        double v = std::round(C[k / 8][k % 8] / qv);
                        v = std::min(std::max(v, -32767.0), 32767.0);
                        coefs[64 * b + k] = int16_t(v);
                    }
                }
                streams[s] = encode_component(coefs.data(), g.log2);
            }
            const std::vector<uint8_t>* p4[4] = {&streams[0], &streams[1], &streams[2], &streams[3]};
            tiles[idx] = make_tile(qs, p4);
            if (tiles[idx].size() > 65535 || streams[0].size() > 65535 || streams[1].size() > 65535 ||
                streams[2].size() > 65535)
                too_big = true;
        }
    });
    if (too_big) return 0;
    auto pkt = frame_packet(spec, tiles);
    if (pkt.size() > cap) return pkt.size();
    std::memcpy(out, pkt.data(), pkt.size());
    return pkt.size();
}

size_t prs_corrupt_tiles(uint8_t* pkt, size_t len, float fraction, uint64_t seed, uint64_t* tiles,
                         size_t cap) {
    if (len < 10 + 70) return 0;
    size_t body_end = 10 + size_t(be16(pkt + 8)) - 2;
    const uint8_t* body = pkt + 10;
    size_t w = be16(body + 6), h = be16(body + 8);
    uint32_t alignment = (be16(body + 68) >> 1) & 7;
    auto row = grid_row(w, alignment);
    size_t ntiles = row.size() * ((h + 15) / 16);
    size_t off = body_end + 2 * ntiles;
    Rng rng{prs_rng_new(seed)};
    const uint32_t thresh = uint32_t(std::min(1.0, double(fraction)) * 4294967295.0);
    size_t n = 0;
    for (size_t i = 0; i < ntiles; i++) {
        size_t size = be16(pkt + body_end + 2 * i);
        uint8_t* t = pkt + off;
        off += size;
        if (rng.next_u32() >= thresh || size < 12 || off > len) continue;
        if (n < cap) tiles[n] = i;
        n++;
        if (rng.below(2) == 0) {
            // Invalid tile header: one of Apple's rejection rules.
            switch (rng.below(4)) {
                case 0: t[1] = 0; break;               // qscale 0
                case 1: t[0] = uint8_t(7 << 3); break;  // header shorter than 8
                case 2: set_be16(t + 2 + 2 * rng.below(3), 0); break;  // empty stream
                default: set_be16(t + 6, uint16_t(size)); break;       // streams overrun the tile
            }
        } else {
            // Malformed stream bytes: the tile decodes, deterministically.
            uint32_t flips = 1 + rng.below(8);
            for (uint32_t k = 0; k < flips; k++) {
                size_t at = 8 + rng.below(uint32_t(size - 8));
                t[at] = uint8_t(rng.next_u32());
            }
        }
    }
    return n;
}

}  // extern "C"
