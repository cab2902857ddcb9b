// dng.cpp -- one decoded frame as a DNG file: the container and tags of the
// crate's DNG export (examples/prr2dng/dng.rs, tiff.rs, colour.rs), host
// C++ of libprr.so. The image data (uncompressed visible samples, or the
// lossless JPEG tiles the device encodes) comes in as chunks; this file
// writes the little-endian TIFF around them, with one IFD whose tags are
// the crate's, value for value.

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <new>
#include <string>
#include <vector>

#include "../../include/prr.h"
#include "context.h"

struct prr_dng_file {
    std::vector<uint8_t> data;
};

namespace prr {
namespace dng {
namespace {

// --- TIFF (tiff.rs) ---------------------------------------------------------

struct Value {
    uint16_t kind;  // TIFF field type: 1 byte, 2 ascii, 3 short, 4 long, 5 rational, 10 srational
    uint32_t count;
    std::vector<uint8_t> bytes;  // little-endian
};

void le16(std::vector<uint8_t>& o, uint32_t v) {
    o.push_back(uint8_t(v));
    o.push_back(uint8_t(v >> 8));
}
void le32(std::vector<uint8_t>& o, uint32_t v) {
    for (int i = 0; i < 4; i++) o.push_back(uint8_t(v >> (8 * i)));
}

Value bytes(const std::vector<uint8_t>& v) { return Value{1, uint32_t(v.size()), v}; }
Value ascii(const std::string& s) {
    Value v{2, uint32_t(s.size() + 1), std::vector<uint8_t>(s.begin(), s.end())};
    v.bytes.push_back(0);
    return v;
}
Value shorts(const std::vector<uint32_t>& xs) {
    Value v{3, uint32_t(xs.size()), {}};
    for (uint32_t x : xs) le16(v.bytes, x);
    return v;
}
Value longs(const std::vector<uint32_t>& xs) {
    Value v{4, uint32_t(xs.size()), {}};
    for (uint32_t x : xs) le32(v.bytes, x);
    return v;
}
Value rationals(const std::vector<std::pair<uint32_t, uint32_t>>& xs) {
    Value v{5, uint32_t(xs.size()), {}};
    for (auto& x : xs) le32(v.bytes, x.first), le32(v.bytes, x.second);
    return v;
}
Value srationals(const std::vector<std::pair<int32_t, int32_t>>& xs) {
    Value v{10, uint32_t(xs.size()), {}};
    for (auto& x : xs) le32(v.bytes, uint32_t(x.first)), le32(v.bytes, uint32_t(x.second));
    return v;
}

// Value::srational (tiff.rs:62-79): the closest signed rational with a
// power-of-ten denominator of at most 10^6.
std::pair<int32_t, int32_t> srational(double v) {
    int64_t d = 1000000;
    while (d > 1 && std::fabs(v * double(d)) >= double(INT32_MAX)) d /= 10;
    const double n = std::round(v * double(d));
    if (std::isnan(n)) return {0, int32_t(d)};
    const double c = std::fmin(std::fmax(n, double(INT32_MIN)), double(INT32_MAX));
    return {int32_t(c), int32_t(d)};
}

// Value::rational (tiff.rs:81-98), for non-negative values.
std::pair<uint32_t, uint32_t> rational(double v) {
    uint64_t d = 1000000;
    while (d > 1 && v * double(d) >= double(UINT32_MAX)) d /= 10;
    const double n = std::round(v * double(d));
    if (std::isnan(n)) return {0, uint32_t(d)};
    const double c = std::fmin(std::fmax(n, 0.0), double(UINT32_MAX));
    return {uint32_t(c), uint32_t(d)};
}

constexpr uint16_t kStripOffsets = 273, kRowsPerStrip = 278, kStripByteCounts = 279;
constexpr uint16_t kTileWidth = 322, kTileLength = 323, kTileOffsets = 324, kTileByteCounts = 325;

// tiff::write (tiff.rs:117-187) up to the image data: the header, the IFD
// (entries by tag) and the values too large for their entry (each padded to
// an even length). The chunks follow it, each padded to an even length, at
// the offsets the layout tags give.
std::vector<uint8_t> tiff_prefix(std::map<uint16_t, Value> tags, bool tiles, uint32_t rows_or_width,
                                 uint32_t tile_height, const std::vector<uint32_t>& sizes) {
    uint16_t offsets_tag, counts_tag;
    if (!tiles) {
        tags[kRowsPerStrip] = longs({rows_or_width});
        offsets_tag = kStripOffsets, counts_tag = kStripByteCounts;
    } else {
        tags[kTileWidth] = longs({rows_or_width});
        tags[kTileLength] = longs({tile_height});
        offsets_tag = kTileOffsets, counts_tag = kTileByteCounts;
    }
    tags[counts_tag] = longs(sizes);
    tags[offsets_tag] = longs(std::vector<uint32_t>(sizes.size(), 0));
    const size_t ifd_size = 2 + 12 * tags.size() + 4;
    size_t values_size = 0;
    for (const auto& kv : tags) {
        const size_t len = kv.second.bytes.size();
        if (len > 4) values_size += len + (len & 1);
    }
    uint32_t offset = uint32_t(8 + ifd_size + values_size);
    std::vector<uint32_t> offsets;
    for (uint32_t n : sizes) {
        offsets.push_back(offset);
        offset += n + (n & 1);
    }
    tags[offsets_tag] = longs(offsets);

    std::vector<uint8_t> out;
    out.reserve(8 + ifd_size + values_size);
    out.push_back('I');
    out.push_back('I');
    le16(out, 42);
    le32(out, 8);
    le16(out, uint32_t(tags.size()));
    std::vector<uint8_t> overflow;
    const size_t values_start = 8 + ifd_size;
    for (const auto& kv : tags) {
        const Value& v = kv.second;
        le16(out, kv.first);
        le16(out, v.kind);
        le32(out, v.count);
        if (v.bytes.size() <= 4) {
            uint8_t inl[4] = {0, 0, 0, 0};
            std::memcpy(inl, v.bytes.data(), v.bytes.size());
            out.insert(out.end(), inl, inl + 4);
        } else {
            le32(out, uint32_t(values_start + overflow.size()));
            overflow.insert(overflow.end(), v.bytes.begin(), v.bytes.end());
            if (v.bytes.size() & 1) overflow.push_back(0);
        }
    }
    le32(out, 0);  // no further IFD
    out.insert(out.end(), overflow.begin(), overflow.end());
    return out;
}

// --- colour (colour.rs) -----------------------------------------------------

struct M3 {
    double m[3][3];
};
struct V3 {
    double v[3];
};
struct XY {
    double x, y;
};

const XY kD65{0.31271, 0.32902};
const XY kD50{0.34567, 0.35850};
const M3 kBradford{{{0.8951, 0.2664, -0.1614}, {-0.7502, 1.7135, 0.0367}, {0.0389, -0.0685, 1.0296}}};
const struct {
    uint16_t code;
    double t;
} kIlluminants[5] = {{17, 2856.0}, {23, 5003.0}, {20, 5503.0}, {21, 6504.0}, {22, 7504.0}};

M3 mul(const M3& a, const M3& b) {
    M3 r;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) r.m[i][j] = a.m[i][0] * b.m[0][j] + a.m[i][1] * b.m[1][j] + a.m[i][2] * b.m[2][j];
    return r;
}
V3 apply(const M3& m, const V3& v) {
    V3 r;
    for (int i = 0; i < 3; i++) r.v[i] = m.m[i][0] * v.v[0] + m.m[i][1] * v.v[1] + m.m[i][2] * v.v[2];
    return r;
}
M3 diag(const V3& v) { return M3{{{v.v[0], 0.0, 0.0}, {0.0, v.v[1], 0.0}, {0.0, 0.0, v.v[2]}}}; }
// The inverse by cofactors (colour.rs:171-179).
M3 inverse(const M3& a) {
    auto cof = [&](int r, int c) {
        const int r0 = (r + 1) % 3, r1 = (r + 2) % 3, c0 = (c + 1) % 3, c1 = (c + 2) % 3;
        return a.m[r0][c0] * a.m[r1][c1] - a.m[r0][c1] * a.m[r1][c0];
    };
    const double det = a.m[0][0] * cof(0, 0) + a.m[0][1] * cof(0, 1) + a.m[0][2] * cof(0, 2);
    M3 r;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) r.m[i][j] = cof(j, i) / det;
    return r;
}
V3 xyz(XY w) { return V3{{w.x / w.y, 1.0, (1.0 - w.x - w.y) / w.y}}; }

// Krystek's Planckian locus in CIE 1960 uv (colour.rs:151-159).
XY planck_xy(double t) {
    const double u = (0.860117757 + 1.54118254e-4 * t + 1.28641212e-7 * t * t) /
                     (1.0 + 8.42420235e-4 * t + 7.08145163e-7 * t * t);
    const double v = (0.317398726 + 4.22806245e-5 * t + 4.20481691e-8 * t * t) /
                     (1.0 - 2.89741816e-5 * t + 1.61456053e-7 * t * t);
    const double d = 2.0 * u - 8.0 * v + 4.0;
    return XY{3.0 * u / d, 2.0 * v / d};
}
// The CIE daylight locus (colour.rs:162-173); t^3 and t^2 by multiplication.
XY daylight_xy(double t) {
    if (t == 6500.0 || t == 6504.0) return kD65;
    const double t2 = t * t, t3 = t * t2;
    const double x = t <= 7000.0 ? -4.6070e9 / t3 + 2.9678e6 / t2 + 0.09911e3 / t + 0.244063
                                 : -2.0064e9 / t3 + 1.9018e6 / t2 + 0.24748e3 / t + 0.237040;
    return XY{x, -3.0 * x * x + 2.870 * x - 0.275};
}
XY white_xy(double t) { return t < 4000.0 ? planck_xy(t) : daylight_xy(t); }
// Bradford adaptation from white `from` to white `to` (colour.rs:151-156).
M3 bradford(XY from, XY to) {
    const V3 s = apply(kBradford, xyz(from)), d = apply(kBradford, xyz(to));
    const V3 gains{{d.v[0] / s.v[0], d.v[1] / s.v[1], d.v[2] / s.v[2]}};
    return mul(mul(inverse(kBradford), diag(gains)), kBradford);
}

double gain(float g) { return g > 0.0f && std::isfinite(g) ? double(g) : 1.0; }

// DngColour::new (colour.rs:74-111).
prr_dng_colour colour_of(const prr_header& h) {
    prr_dng_colour c{};
    const double temperature = h.wb_cct == 0 ? 6504.0 : std::fmin(std::fmax(double(h.wb_cct), 1000.0), 25000.0);
    const V3 wb{{gain(h.wb_red), 1.0, gain(h.wb_blue)}};
    M3 m;
    for (int i = 0; i < 9; i++) m.m[i / 3][i % 3] = double(h.color_matrix[i]);
    const XY white = white_xy(temperature);
    const M3 camera_to_scene = mul(mul(bradford(kD65, white), m), diag(wb));
    const M3 cm = inverse(camera_to_scene);
    const V3 n = apply(cm, xyz(white));
    double largest = -1.7976931348623157e308;
    for (double v : n.v) largest = std::fmax(largest, v);
    int best = 0;
    for (int k = 1; k < 5; k++) {
        const double dk = std::fabs(1.0 / kIlluminants[k].t - 1.0 / temperature);
        const double db = std::fabs(1.0 / kIlluminants[best].t - 1.0 / temperature);
        if (dk < db) best = k;
    }
    const M3 fm = mul(bradford(kD65, kD50), m);
    c.temperature = temperature;
    c.illuminant = kIlluminants[best].code;
    for (int i = 0; i < 9; i++) {
        c.color_matrix[i] = cm.m[i / 3][i % 3] / largest;
        c.forward_matrix[i] = fm.m[i / 3][i % 3];
    }
    for (int i = 0; i < 3; i++) c.as_shot_neutral[i] = 1.0 / wb.v[i];
    c.baseline_exposure = std::log2(gain(h.gain));
    return c;
}

// --- the DNG tags (dng.rs:138-209) ------------------------------------------

// Curve::linearize (src/curve.rs:14-24).
uint16_t linearize(const uint16_t* curve, uint32_t code) {
    const uint32_t seg = code >> 13, frac = code & 0x1FFF;
    const uint32_t c0 = curve[seg], c1 = seg + 1 < 8 ? curve[seg + 1] : 65536u;
    const uint32_t delta = (c1 - c0) & 0xFFFF;
    const uint32_t out = (c0 * 8192 + delta * frac + 4096) >> 13;
    return uint16_t(out < 65535 ? out : 65535);
}

std::string escape_ascii(const uint8_t* k, size_t n) {
    static const char* hex = "0123456789abcdef";
    std::string s;
    for (size_t i = 0; i < n; i++) {
        const uint8_t b = k[i];
        switch (b) {
            case '\t': s += "\\t"; break;
            case '\r': s += "\\r"; break;
            case '\n': s += "\\n"; break;
            case '\\': s += "\\\\"; break;
            case '\'': s += "\\'"; break;
            case '"': s += "\\\""; break;
            default:
                if (b >= 0x20 && b < 0x7f) {
                    s += char(b);
                } else {
                    s += "\\x";
                    s += hex[b >> 4];
                    s += hex[b & 15];
                }
        }
    }
    return s;
}

const char* const kSoftware = "proresraw_rs prr2dng 0.1.0";

std::map<uint16_t, Value> tags(const prr_header& h, const prr_dng_clip& clip, int samples) {
    const prr_dng_colour colour = colour_of(h);
    const uint32_t width = h.width, height = h.height;
    std::map<uint16_t, Value> t;
    t[254] = longs({0});  // NewSubFileType: main image
    t[256] = longs({width});
    t[257] = longs({height});
    t[258] = shorts({16});     // BitsPerSample
    t[262] = shorts({32803});  // PhotometricInterpretation: CFA
    if (clip.make) t[271] = ascii(clip.make);
    if (clip.model) t[272] = ascii(clip.model);
    t[274] = shorts({clip.orientation ? clip.orientation : 1u});
    t[277] = shorts({1});  // SamplesPerPixel
    t[284] = shorts({1});  // PlanarConfiguration: chunky
    t[305] = ascii(clip.software ? clip.software : kSoftware);
    if (clip.date_time) t[306] = ascii(clip.date_time);
    t[33421] = shorts({2, 2});  // CFARepeatPatternDim
    // CFAPattern: red 0, green 1, blue 2 at (0,0), (0,1), (1,0), (1,1).
    const uint32_t rr = (h.bayer_pattern >> 1) & 1, rc = h.bayer_pattern & 1;
    std::vector<uint8_t> cfa;
    for (uint32_t r = 0; r < 2; r++)
        for (uint32_t c = 0; c < 2; c++)
            cfa.push_back(r == rr && c == rc ? 0 : (r == (rr ^ 1) && c == (rc ^ 1) ? 2 : 1));
    t[33422] = bytes(cfa);
    t[50706] = bytes({1, 4, 0, 0});  // DNGVersion
    t[50707] = bytes({1, 3, 0, 0});  // DNGBackwardVersion
    // UniqueCameraModel (dng.rs:59-73): make and model joined by a space.
    std::string camera;
    if (clip.make) camera = clip.make;
    if (clip.model) camera = clip.make ? camera + " " + clip.model : std::string(clip.model);
    t[50708] = ascii(camera.empty() ? "ProRes RAW " + escape_ascii(h.vendor, 4) : camera + " (ProRes RAW)");
    t[50710] = bytes({0, 1, 2});  // CFAPlaneColor
    t[50711] = shorts({1});       // CFALayout: rectangular
    if (samples == PRR_DNG_CODE_VALUES) {
        std::vector<uint32_t> lut(65536);
        for (uint32_t code = 0; code < 65536; code++) lut[code] = linearize(h.curve, code);
        t[50712] = shorts(lut);  // LinearizationTable
    }
    t[50713] = shorts({1, 1});      // BlackLevelRepeatDim
    t[50714] = longs({256});        // BlackLevel
    t[50717] = longs({h.white_level});
    const uint32_t cl = h.crop[0], cr = h.crop[1], ct = h.crop[2], cb = h.crop[3];
    const uint32_t crop_w = width > cl + cr ? width - (cl + cr) : 0;
    const uint32_t crop_h = height > ct + cb ? height - (ct + cb) : 0;
    if (crop_w > 0 && crop_h > 0) {
        t[50719] = longs({cl, ct});  // DefaultCropOrigin
        t[50720] = longs({crop_w, crop_h});
    }
    std::vector<std::pair<int32_t, int32_t>> cm, fm;
    for (int i = 0; i < 9; i++) cm.push_back(srational(colour.color_matrix[i]));
    for (int i = 0; i < 9; i++) fm.push_back(srational(colour.forward_matrix[i]));
    t[50721] = srationals(cm);  // ColorMatrix1
    std::vector<std::pair<uint32_t, uint32_t>> neutral;
    for (int i = 0; i < 3; i++) neutral.push_back(rational(colour.as_shot_neutral[i]));
    t[50728] = rationals(neutral);                            // AsShotNeutral
    t[50730] = srationals({srational(colour.baseline_exposure)});  // BaselineExposure
    t[50778] = shorts({colour.illuminant});                   // CalibrationIlluminant1
    t[50964] = srationals(fm);                                // ForwardMatrix1
    if (clip.fps_den != 0) t[51044] = srationals({{int32_t(clip.fps_num), int32_t(clip.fps_den)}});  // FrameRate
    return t;
}

}  // namespace
}  // namespace dng

constexpr uint32_t kDngTile = 256;  // dng.rs:23-25

// dng::write (dng.rs:77-111) up to the image data, for chunks (one strip of
// the visible samples, or the tiles' streams in order) of `sizes` bytes.
int dng_prefix(const prr_header* header, const prr_dng_clip* clip, int samples, int compression,
               const std::vector<uint32_t>& sizes, std::vector<uint8_t>& prefix) {
    if (!header || (samples != PRR_DNG_CODE_VALUES && samples != PRR_DNG_LINEAR) ||
        (compression != PRR_DNG_UNCOMPRESSED && compression != PRR_DNG_LJ92))
        return PRR_ERR_INVALID;
    const prr_dng_clip none{};
    const prr_dng_clip& c = clip ? *clip : none;
    if (c.orientation > 8) return PRR_ERR_INVALID;
    try {
        auto t = dng::tags(*header, c, samples);
        if (compression == PRR_DNG_UNCOMPRESSED) {
            if (sizes.size() != 1) return PRR_ERR_INVALID;
            t[259] = dng::shorts({1});
            prefix = dng::tiff_prefix(std::move(t), false, header->height, 0, sizes);
        } else {
            const size_t across = (header->width + kDngTile - 1) / kDngTile;
            const size_t down = (header->height + kDngTile - 1) / kDngTile;
            if (sizes.size() != across * down) return PRR_ERR_INVALID;
            t[259] = dng::shorts({7});
            prefix = dng::tiff_prefix(std::move(t), true, kDngTile, kDngTile, sizes);
        }
        return PRR_OK;
    } catch (const std::bad_alloc&) {
        return PRR_ERR_NO_MEMORY;
    }
}

// The whole file around chunks already in host memory.
int dng_assemble(const prr_header* header, const prr_dng_clip* clip, int samples, int compression,
                 const uint8_t* data, const uint64_t* offsets, size_t nchunks, prr_dng_file** out) {
    if (!out || (nchunks > 0 && (!data || !offsets))) return PRR_ERR_INVALID;
    *out = nullptr;
    std::vector<uint32_t> sizes;
    for (size_t i = 0; i < nchunks; i++) {
        if (offsets[i + 1] < offsets[i] || offsets[i + 1] - offsets[i] > 0xFFFFFFFFull) return PRR_ERR_INVALID;
        sizes.push_back(uint32_t(offsets[i + 1] - offsets[i]));
    }
    std::vector<uint8_t> prefix;
    PRR_TRY(dng_prefix(header, clip, samples, compression, sizes, prefix));
    try {
        auto* f = new prr_dng_file;
        size_t total = prefix.size();
        for (uint32_t n : sizes) total += n + (n & 1);
        f->data.reserve(total);
        f->data.insert(f->data.end(), prefix.begin(), prefix.end());
        for (size_t i = 0; i < nchunks; i++) {
            f->data.insert(f->data.end(), data + offsets[i], data + offsets[i + 1]);
            if (sizes[i] & 1) f->data.push_back(0);
        }
        *out = f;
        return PRR_OK;
    } catch (const std::bad_alloc&) {
        return PRR_ERR_NO_MEMORY;
    }
}

prr_dng_file* dng_file_new(size_t bytes) {
    auto* f = new prr_dng_file;
    f->data.resize(bytes);
    return f;
}
uint8_t* dng_file_bytes(prr_dng_file* f) { return f->data.data(); }

}  // namespace prr

extern "C" {

int prr_dng_assemble(const prr_header* header, const prr_dng_clip* clip, int samples, int compression,
                     const uint8_t* data, const uint64_t* offsets, size_t nchunks, prr_dng_file** out) {
    return prr::dng_assemble(header, clip, samples, compression, data, offsets, nchunks, out);
}

const uint8_t* prr_dng_data(const prr_dng_file* f, size_t* len) {
    if (!f) return nullptr;
    if (len) *len = f->data.size();
    return f->data.data();
}

void prr_dng_free(prr_dng_file* f) { delete f; }

int prr_dng_colour_of(const prr_header* header, prr_dng_colour* out) {
    if (!header || !out) return PRR_ERR_INVALID;
    *out = prr::dng::colour_of(*header);
    return PRR_OK;
}

int prr_dng_srational(double v, int32_t* num, int32_t* den) {
    if (!num || !den) return PRR_ERR_INVALID;
    const auto r = prr::dng::srational(v);
    *num = r.first, *den = r.second;
    return PRR_OK;
}

int prr_dng_rational(double v, uint32_t* num, uint32_t* den) {
    if (!num || !den) return PRR_ERR_INVALID;
    const auto r = prr::dng::rational(v);
    *num = r.first, *den = r.second;
    return PRR_OK;
}

// quicktime_date_time (dng.rs:211-232): days from 1904-01-01 to the Unix
// epoch, then the civil date of a Unix day (Howard Hinnant's algorithm).
int prr_dng_date_time(uint64_t seconds, char out[20]) {
    if (!out) return PRR_ERR_INVALID;
    const int64_t days = int64_t(seconds / 86400);
    const uint64_t time = seconds % 86400;
    const int64_t z = days - 24107 + 719468;
    const int64_t era = (z >= 0 ? z : z - 146096) / 146097;
    const int64_t doe = z - era * 146097;
    const int64_t yoe = (doe - doe / 1460 + doe / 36524 - doe / 146096) / 365;
    const int64_t doy = doe - (365 * yoe + yoe / 4 - yoe / 100);
    const int64_t mp = (5 * doy + 2) / 153;
    const int64_t day = doy - (153 * mp + 2) / 5 + 1;
    const int64_t month = mp < 10 ? mp + 3 : mp - 9;
    const int64_t year = yoe + era * 400 + (month <= 2 ? 1 : 0);
    // The crate's text has 19 characters while the year has four digits;
    // a later year does not fit the 20-byte result.
    char text[64];
    const int n = std::snprintf(text, sizeof(text), "%04lld:%02lld:%02lld %02llu:%02llu:%02llu", (long long)year,
                                (long long)month, (long long)day, (unsigned long long)(time / 3600),
                                (unsigned long long)(time / 60 % 60), (unsigned long long)(time % 60));
    if (n != 19) return PRR_ERR_BUFFER;
    std::memcpy(out, text, 20);
    return PRR_OK;
}

}  // extern "C"
