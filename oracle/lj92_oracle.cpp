// lj92_oracle.cpp -- CPU restatement of the DNG export's lossless JPEG
// encoder (examples/prr2dng/lj92.rs) and tile cut (examples/prr2dng/dng.rs).
// TEST INFRASTRUCTURE ONLY: see lj92_oracle.h.

#include "lj92_oracle.h"

#include <algorithm>
#include <atomic>
#include <cstring>
#include <thread>
#include <vector>

namespace {

// The magnitude category SSSS of a difference: its bit length (lj92.rs:90-93).
int category(int32_t d) {
    const uint32_t a = d < 0 ? uint32_t(-int64_t(d)) : uint32_t(d);
    return a == 0 ? 0 : 32 - __builtin_clz(a);
}

// Prediction differences in coding order (lj92.rs:72-86): predictor 1 (the
// sample `components` to the left), the sample above for a row's first
// pixel, half the range for the image's first; modulo 2^16, centred on 0.
std::vector<int32_t> differences(const uint16_t* s, size_t width, size_t height, size_t components) {
    std::vector<int32_t> d(width * height);
    for (size_t i = 0; i < width * height; i++) {
        const size_t row = i / width, column = i % width;
        uint16_t prediction;
        if (column >= components)
            prediction = s[i - components];
        else if (row > 0)
            prediction = s[i - width];
        else
            prediction = 1 << 15;
        d[i] = int16_t(uint16_t(s[i] - prediction));
    }
    return d;
}

struct Table {
    uint8_t counts[16];
    uint8_t values[17];
    int nvalues;
    uint16_t code[17];
    uint8_t length[17];
};

// ITU T.81 Annex K.2 with a reserved all-ones code (lj92.rs:96-202).
Table optimal(const uint64_t* histogram) {
    const int kReserved = 17;
    uint64_t freq[18];
    for (int v = 0; v < 17; v++) freq[v] = histogram[v];
    freq[kReserved] = 1;
    int size[18] = {0};
    int others[18];
    for (int& o : others) o = -1;
    for (;;) {
        // The two least frequent symbols left; ties go to the larger symbol.
        int least = -1, second = -1;
        for (int v = 0; v < 18; v++) {
            if (freq[v] == 0) continue;
            if (least < 0 || freq[v] <= freq[least]) {
                second = least;
                least = v;
            } else if (second < 0 || freq[v] <= freq[second]) {
                second = v;
            }
        }
        if (least < 0 || second < 0) break;
        const int v1 = least, v2 = second;
        freq[v1] += freq[v2];
        freq[v2] = 0;
        int v = v1;
        for (;;) {
            size[v]++;
            if (others[v] < 0) break;
            v = others[v];
        }
        others[v] = v2;
        v = v2;
        for (;;) {
            size[v]++;
            if (others[v] < 0) break;
            v = others[v];
        }
    }
    // Codes per length, then lengths limited to 16 (Figure K.3).
    uint32_t bits[33] = {0};
    for (int s : size)
        if (s > 0) bits[s]++;
    for (int i = 32; i > 16; i--) {
        while (bits[i] > 0) {
            int j = i - 2;
            while (bits[j] == 0) j--;
            bits[i] -= 2;
            bits[i - 1] += 1;
            bits[j + 1] += 2;
            bits[j] -= 1;
        }
    }
    // The reserved symbol's code, the longest, is dropped.
    int i = 16;
    while (bits[i] == 0) i--;
    bits[i]--;

    Table t{};
    int order[17], n = 0;
    for (int v = 0; v < 17; v++)
        if (size[v] > 0) order[n++] = v;
    std::stable_sort(order, order + n, [&](int a, int b) { return size[a] != size[b] ? size[a] < size[b] : a < b; });
    for (int k = 0; k < 16; k++) t.counts[k] = uint8_t(bits[k + 1]);
    for (int k = 0; k < n; k++) t.values[k] = uint8_t(order[k]);
    t.nvalues = n;
    // Canonical codes from the counts (Annex C).
    uint32_t code = 0;
    int k = 0;
    for (int length = 1; length <= 16; length++) {
        for (int c = 0; c < t.counts[length - 1]; c++) {
            t.code[t.values[k]] = uint16_t(code);
            t.length[t.values[k]] = uint8_t(length);
            code++;
            k++;
        }
        code <<= 1;
    }
    return t;
}

// Entropy-coded bits, most significant first, 0xFF bytes stuffed with 0x00
// (lj92.rs:209-246).
struct BitWriter {
    std::vector<uint8_t>& out;
    uint64_t buffer = 0;
    uint32_t count = 0;
    void put(uint64_t value, uint32_t length) {
        buffer = (buffer << length) | value;
        count += length;
        while (count >= 8) {
            count -= 8;
            const uint8_t byte = uint8_t(buffer >> count);
            out.push_back(byte);
            if (byte == 0xFF) out.push_back(0);
        }
        buffer &= (uint64_t(1) << count) - 1;
    }
    void finish() {
        if (count > 0) {
            const uint32_t pad = 8 - count;
            put((uint64_t(1) << pad) - 1, pad);
        }
    }
};

void be16(std::vector<uint8_t>& o, uint32_t v) {
    o.push_back(uint8_t(v >> 8));
    o.push_back(uint8_t(v));
}

std::vector<uint8_t> encode(const uint16_t* samples, size_t width, size_t height, size_t components) {
    const std::vector<int32_t> d = differences(samples, width, height, components);
    uint64_t histogram[17] = {0};
    for (int32_t x : d) histogram[category(x)]++;
    const Table t = optimal(histogram);
    std::vector<uint8_t> out;
    out.reserve(width * height * 2 + 1024);
    out.push_back(0xFF);  // SOI
    out.push_back(0xD8);
    out.push_back(0xFF);  // SOF3: lossless, Huffman, 16-bit
    out.push_back(0xC3);
    be16(out, uint32_t(8 + 3 * components));
    out.push_back(16);
    be16(out, uint32_t(height));
    be16(out, uint32_t(width / components));
    out.push_back(uint8_t(components));
    for (size_t id = 0; id < components; id++) {
        out.push_back(uint8_t(id));
        out.push_back(0x11);
        out.push_back(0);
    }
    out.push_back(0xFF);  // DHT: one DC table, class 0, id 0
    out.push_back(0xC4);
    be16(out, uint32_t(2 + 1 + 16 + t.nvalues));
    out.push_back(0);
    out.insert(out.end(), t.counts, t.counts + 16);
    out.insert(out.end(), t.values, t.values + t.nvalues);
    out.push_back(0xFF);  // SOS: table 0 for every component, predictor 1
    out.push_back(0xDA);
    be16(out, uint32_t(6 + 2 * components));
    out.push_back(uint8_t(components));
    for (size_t id = 0; id < components; id++) {
        out.push_back(uint8_t(id));
        out.push_back(0);
    }
    out.push_back(1);
    out.push_back(0);
    out.push_back(0);
    BitWriter bits{out};
    for (int32_t x : d) {
        const int ssss = category(x);
        bits.put(t.code[ssss], t.length[ssss]);
        // Category 16 (the difference 32768) has no extra bits; negative
        // differences go as d - 1 in ssss bits.
        if (ssss > 0 && ssss < 16) {
            const int32_t extra = x < 0 ? x - 1 : x;
            bits.put(uint64_t(uint32_t(extra)) & ((uint64_t(1) << ssss) - 1), uint32_t(ssss));
        }
    }
    bits.finish();
    out.push_back(0xFF);  // EOI
    out.push_back(0xD9);
    return out;
}

// dng::tile's clamp: past the edge, the last row or column of the same phase.
size_t clamp(size_t i, size_t n) { return i < n ? i : n - 2 + (i - n) % 2; }

}  // namespace

extern "C" {

int orc_lj92_encode(const uint16_t* samples, size_t width, size_t height, size_t components, uint8_t* out,
                    size_t cap, size_t* len) {
    if (!samples || !len || components == 0 || width % components != 0) return -1;
    const std::vector<uint8_t> s = encode(samples, width, height, components);
    *len = s.size();
    if (s.size() > cap || !out) return -1;
    std::memcpy(out, s.data(), s.size());
    return 0;
}

void orc_lj92_huffman(const uint64_t histogram[17], uint8_t counts[16], uint8_t values[17], int* nvalues,
                      uint16_t codes[17], uint8_t lengths[17]) {
    const Table t = optimal(histogram);
    std::memcpy(counts, t.counts, 16);
    std::memcpy(values, t.values, 17);
    *nvalues = t.nvalues;
    std::memcpy(codes, t.code, sizeof(t.code));
    std::memcpy(lengths, t.length, sizeof(t.length));
}

int orc_dng_tile(const uint16_t* values, size_t width, size_t height, size_t stride, size_t left, size_t top,
                 size_t tile, uint16_t* out) {
    if (!values || !out || width < 2 || height < 2 || stride < width) return -1;
    for (size_t y = 0; y < tile; y++) {
        const uint16_t* row = values + clamp(top + y, height) * stride;
        for (size_t x = 0; x < tile; x++) out[y * tile + x] = row[clamp(left + x, width)];
    }
    return 0;
}

int orc_lj92_tiles(const uint16_t* values, size_t width, size_t height, size_t stride, size_t tile, int threads,
                   uint8_t* out, size_t cap, uint64_t* offsets) {
    if (!values || !offsets || width < 2 || height < 2 || tile == 0 || tile % 2 != 0) return -1;
    const size_t across = (width + tile - 1) / tile, down = (height + tile - 1) / tile;
    const size_t n = across * down;
    std::vector<std::vector<uint8_t>> streams(n);
    std::atomic<size_t> next{0};
    auto work = [&] {
        std::vector<uint16_t> t(tile * tile);
        for (size_t i = next++; i < n; i = next++) {
            orc_dng_tile(values, width, height, stride, i % across * tile, i / across * tile, tile, t.data());
            streams[i] = encode(t.data(), tile, tile, 2);
        }
    };
    const int nt = threads > 0 ? threads : int(std::max(1u, std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    for (int k = 1; k < nt; k++) pool.emplace_back(work);
    work();
    for (auto& th : pool) th.join();
    uint64_t total = 0;
    for (size_t i = 0; i < n; i++) {
        offsets[i] = total;
        total += streams[i].size();
    }
    offsets[n] = total;
    if (total > cap || !out) return -1;
    for (size_t i = 0; i < n; i++) std::memcpy(out + offsets[i], streams[i].data(), streams[i].size());
    return 0;
}

}  // extern "C"
