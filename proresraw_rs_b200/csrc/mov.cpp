// mov.cpp -- the sample table of one video track of a QuickTime (or ISO base
// media) movie: where each presented frame's bytes are, the frame rate and
// the movie's text metadata (src/mov.rs). Host code of libprr.so, the step
// before the decoders: its samples are the packets a batch decodes. Only the
// `moov` atom is read into memory; samples are read with positional reads,
// so one open track serves every decoding thread without a lock.
//
// Messages name the atom or structure at fault with their context, as the
// crate's do, so that a caller sees the same text.

#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cerrno>
#include <charconv>
#include <cstdint>
#include <cstring>
#include <map>
#include <optional>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/prr.h"

namespace prr {
namespace mov {
namespace {

struct Error : std::runtime_error {
    using std::runtime_error::runtime_error;
};

#define MOV_ENSURE(cond, message)          \
    do {                                   \
        if (!(cond)) throw Error(message); \
    } while (0)

constexpr uint64_t kMaxMoov = 64ull << 20;     // larger `moov` atoms are refused (src/mov.rs:84)
constexpr uint64_t kMaxSamples = 10000000ull;  // src/mov.rs:86
const char* const kFirstAtoms[] = {"ftyp", "moov", "mdat", "wide", "free", "skip", "pnot"};

struct Span {
    const uint8_t* p = nullptr;
    size_t n = 0;
    Span sub(size_t a, size_t b) const { return Span{p + a, b - a}; }
};

struct Atom {
    uint8_t kind[4];
    Span body;
    bool is(const char* k) const { return std::memcmp(kind, k, 4) == 0; }
};

using Kind = const uint8_t*;

// A fourcc for messages, bytes escaped as Rust's escape_ascii does.
std::string name(const uint8_t* k) {
    static const char* hex = "0123456789abcdef";
    std::string s;
    for (int i = 0; i < 4; i++) {
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
std::string name(const char* k) { return name(reinterpret_cast<const uint8_t*>(k)); }

// A float as Rust's Display prints it: the shortest decimal that reads back
// to the same value, without an exponent.
std::string decimal(double v) {
    char buf[400];
    const auto r = std::to_chars(buf, buf + sizeof(buf), v, std::chars_format::fixed);
    return std::string(buf, r.ptr);
}

uint32_t be32(const uint8_t* b) { return uint32_t(b[0]) << 24 | uint32_t(b[1]) << 16 | uint32_t(b[2]) << 8 | b[3]; }
uint64_t be64(const uint8_t* b) { return uint64_t(be32(b)) << 32 | be32(b + 4); }

// `count` entries of `width` bytes at `at` in `kind`'s body (src/mov.rs:730-747).
Span entries(Span body, size_t at, uint64_t count, size_t width, const std::string& kind) {
    const unsigned __int128 bytes = (unsigned __int128)count * width;
    MOV_ENSURE(bytes <= body.n && at <= body.n - size_t(bytes),
               "truncated `" + kind + "` atom: " + std::to_string(count) + " entries do not fit in " +
                   std::to_string(body.n) + " bytes");
    return body.sub(at, at + size_t(bytes));
}
uint32_t u32_at(Span body, size_t at, const std::string& kind) { return be32(entries(body, at, 1, 4, kind).p); }
uint64_t u64_at(Span body, size_t at, const std::string& kind) { return be64(entries(body, at, 1, 8, kind).p); }

// The child atoms of `data` (src/mov.rs:694-719).
std::vector<Atom> children(Span data) {
    std::vector<Atom> atoms;
    Span rest = data;
    while (rest.n > 0) {
        if (rest.n < 8) {
            // QuickTime allows a 32-bit zero after the last child.
            MOV_ENSURE(std::all_of(rest.p, rest.p + rest.n, [](uint8_t b) { return b == 0; }),
                       "truncated atom header");
            break;
        }
        Atom a;
        std::memcpy(a.kind, rest.p + 4, 4);
        uint64_t header, size;
        const uint32_t s32 = be32(rest.p);
        if (s32 == 1) {
            header = 16;
            size = u64_at(rest, 8, name(a.kind));
        } else if (s32 == 0) {
            header = 8;
            size = rest.n;
        } else {
            header = 8;
            size = s32;
        }
        MOV_ENSURE(header <= size && size <= rest.n, "truncated `" + name(a.kind) + "` atom: it claims " +
                                                         std::to_string(size) + " bytes and " +
                                                         std::to_string(rest.n) + " are left");
        a.body = rest.sub(size_t(header), size_t(size));
        atoms.push_back(a);
        rest = rest.sub(size_t(size), rest.n);
    }
    return atoms;
}

const Atom* find(const std::vector<Atom>& atoms, const char* kind) {
    for (const auto& a : atoms)
        if (a.is(kind)) return &a;
    return nullptr;
}

Span require(const std::vector<Atom>& atoms, const char* kind, const std::string& parent) {
    const Atom* a = find(atoms, kind);
    MOV_ENSURE(a, parent + " has no `" + name(kind) + "` atom");
    return a->body;
}

size_t sample_count(uint32_t count) {
    MOV_ENSURE(count <= kMaxSamples, "the video track lists " + std::to_string(count) + " samples, more than the " +
                                         std::to_string(kMaxSamples) + " this reader accepts");
    return count;
}

// The creation time and timescale of a `mvhd` or `mdhd` (src/mov.rs:642-649).
std::pair<uint64_t, uint32_t> times(Span body, const char* kind) {
    MOV_ENSURE(body.n > 0, "truncated `" + name(kind) + "` atom");
    const uint8_t v = body.p[0];
    if (v == 0) return {u32_at(body, 4, kind), u32_at(body, 12, kind)};
    if (v == 1) return {u64_at(body, 4, kind), u32_at(body, 20, kind)};
    throw Error("`" + name(kind) + "` version " + std::to_string(v) + " is not supported");
}

// The orientation of a `tkhd`'s display matrix (src/mov.rs:651-692): only
// the signs of a b c d matter; other matrices show frames as stored.
int orientation(Span tkhd, std::vector<std::string>& warnings) {
    MOV_ENSURE(tkhd.n > 0, "truncated `tkhd` atom");
    const uint8_t v = tkhd.p[0];
    size_t at;
    if (v == 0)
        at = 40;
    else if (v == 1)
        at = 52;
    else
        throw Error("`tkhd` version " + std::to_string(v) + " is not supported");
    auto entry = [&](size_t i) { return double(int32_t(u32_at(tkhd, at + 4 * i, "tkhd"))) / 65536.0; };
    const double a = entry(0), b = entry(1), c = entry(3), d = entry(4);
    auto sign = [](double x) { return int(x > 0.0) - int(x < 0.0); };
    const int sa = sign(a), sb = sign(b), sc = sign(c), sd = sign(d);
    // EXIF values 1..8: identity, mirror horizontal, 180, mirror vertical,
    // transpose, 90 clockwise, transverse, 270.
    if (sa == 1 && sb == 0 && sc == 0 && sd == 1) return 1;
    if (sa == -1 && sb == 0 && sc == 0 && sd == 1) return 2;
    if (sa == -1 && sb == 0 && sc == 0 && sd == -1) return 3;
    if (sa == 1 && sb == 0 && sc == 0 && sd == -1) return 4;
    if (sa == 0 && sb == 1 && sc == 1 && sd == 0) return 5;
    if (sa == 0 && sb == 1 && sc == -1 && sd == 0) return 6;
    if (sa == 0 && sb == -1 && sc == -1 && sd == 0) return 7;
    if (sa == 0 && sb == -1 && sc == 1 && sd == 0) return 8;
    warnings.push_back("the video track's display matrix [" + decimal(a) + " " + decimal(b) + "; " + decimal(c) + " " +
                       decimal(d) + "] is not a quarter turn or mirror, so the frames are shown as stored");
    return 1;
}

// Bytes as text, each maximal ill-formed subsequence replaced by one U+FFFD
// (Unicode's "maximal subpart" practice, as String::from_utf8_lossy): a lead
// byte and the continuation bytes that could still complete it count as one.
std::string lossy_utf8(const uint8_t* p, size_t n) {
    std::string out;
    size_t i = 0;
    while (i < n) {
        const uint8_t b = p[i];
        if (b < 0x80) {
            out += char(b);
            i++;
            continue;
        }
        // Sequence length and the range of the second byte, by lead byte.
        size_t len = 0;
        uint8_t lo = 0x80, hi = 0xBF;
        if (b >= 0xC2 && b <= 0xDF) len = 2;
        else if (b == 0xE0) len = 3, lo = 0xA0;
        else if (b == 0xED) len = 3, hi = 0x9F;
        else if (b >= 0xE1 && b <= 0xEF) len = 3;
        else if (b == 0xF0) len = 4, lo = 0x90;
        else if (b == 0xF4) len = 4, hi = 0x8F;
        else if (b >= 0xF1 && b <= 0xF3) len = 4;
        size_t k = 1;
        if (len > 0) {
            for (; k < len && i + k < n; k++) {
                const uint8_t c = p[i + k];
                const bool in_range = k == 1 ? (c >= lo && c <= hi) : (c >= 0x80 && c <= 0xBF);
                if (!in_range) break;
            }
        }
        if (len > 0 && k == len) {
            out.append(reinterpret_cast<const char*>(p + i), len);
        } else {
            out += "\xEF\xBF\xBD";
        }
        i += k;
    }
    return out;
}

// The UTF-8 items of a `meta` atom whose keys use the `mdta` namespace
// (src/mov.rs:598-640).
std::vector<std::pair<std::string, std::string>> text_metadata(Span meta) {
    Span body;
    if (meta.n >= 8 && std::memcmp(meta.p + 4, "hdlr", 4) == 0) {
        body = meta;  // QuickTime's form: the children follow directly
    } else {
        MOV_ENSURE(meta.n >= 4, "truncated `meta` atom");
        body = meta.sub(4, meta.n);  // ISO's: a version and flags word first
    }
    const auto atoms = children(body);
    const Atom* keys = find(atoms, "keys");
    const Atom* ilst = find(atoms, "ilst");
    std::vector<std::pair<std::string, std::string>> items;
    if (!keys || !ilst) return items;
    const size_t count = u32_at(keys->body, 4, "keys");
    std::vector<std::string> names;
    names.reserve(std::min<size_t>(count, 1024));
    MOV_ENSURE(keys->body.n >= 8, "truncated `keys` atom");
    Span rest = keys->body.sub(8, keys->body.n);
    for (size_t k = 0; k < count; k++) {
        MOV_ENSURE(rest.n >= 4, "truncated `keys` atom");
        const size_t size = std::max<size_t>(be32(rest.p), 8);
        MOV_ENSURE(size <= rest.n, "truncated `keys` atom");
        names.push_back(lossy_utf8(rest.p + 8, size - 8));
        rest = rest.sub(size, rest.n);
    }
    for (const Atom& item : children(ilst->body)) {
        const size_t index = size_t(be32(item.kind)) - 1;  // 1-based key index, wrapping
        if (index >= names.size()) continue;
        for (const Atom& d : children(item.body)) {
            // Type indicator (well-known type 1 is UTF-8), locale, then the value.
            if (d.is("data") && d.body.n >= 8 && be32(d.body.p) == 1) {
                std::string value = lossy_utf8(d.body.p + 8, d.body.n - 8);
                while (!value.empty() && value.back() == '\0') value.pop_back();
                items.emplace_back(names[index], value);
            }
        }
    }
    return items;
}

uint32_t gcd(uint32_t a, uint32_t b) { return b == 0 ? a : gcd(b, a % b); }

// The most common duration, ignoring the last sample, and whether any other
// occurs; ties go to the shorter duration (src/mov.rs:507-518).
std::pair<uint32_t, bool> common_duration(const std::vector<uint32_t>& durations) {
    const size_t body = std::max<size_t>(durations.size() > 0 ? durations.size() - 1 : 0, 1);
    std::map<uint32_t, size_t> counts;
    for (size_t i = 0; i < body && i < durations.size(); i++) counts[durations[i]]++;
    uint32_t mode = 1;
    size_t best = 0;
    for (const auto& kv : counts)  // ascending: the first maximum is the shortest
        if (kv.second > best) {
            best = kv.second;
            mode = kv.first;
        }
    return {mode, counts.size() > 1};
}

struct Sample {
    uint64_t offset;
    uint32_t size;
};

struct Track {
    uint8_t fourcc[4];
    uint32_t fps_num = 0, fps_den = 0;
    bool variable_durations = false;
    std::vector<Sample> samples;
    std::optional<uint64_t> creation_time;
    int orientation = 1;
    std::vector<std::string> warnings;
    std::vector<std::pair<std::string, std::string>> metadata;
};

// The samples the first non-empty edit of `elst` presents (src/mov.rs:522-595).
std::pair<size_t, size_t> edit(Span elst, const std::vector<uint32_t>& durations, uint32_t timescale,
                               uint32_t movie_timescale, std::vector<std::string>& warnings) {
    MOV_ENSURE(elst.n > 0, "truncated `elst` atom");
    const uint8_t version = elst.p[0];
    const size_t count = u32_at(elst, 4, "elst");
    struct E {
        uint64_t duration;
        int64_t time;
        int32_t rate;
    };
    std::vector<E> edits;
    if (version == 0) {
        const Span t = entries(elst, 8, count, 12, "elst");
        for (size_t i = 0; i < count; i++) {
            const uint8_t* e = t.p + 12 * i;
            edits.push_back({be32(e), int64_t(int32_t(be32(e + 4))), int32_t(be32(e + 8))});
        }
    } else if (version == 1) {
        const Span t = entries(elst, 8, count, 20, "elst");
        for (size_t i = 0; i < count; i++) {
            const uint8_t* e = t.p + 20 * i;
            edits.push_back({be64(e), int64_t(be64(e + 8)), int32_t(be32(e + 16))});
        }
    } else {
        throw Error("`elst` version " + std::to_string(version) + " is not supported");
    }
    if (edits.size() > 1)
        warnings.push_back("the video track's edit list has " + std::to_string(edits.size()) +
                           " edits; only the first that shows media is honoured");
    if (!edits.empty() && edits[0].time < 0)
        warnings.push_back("the video track's edit list starts with an empty edit (a delay), which is ignored");
    const E* shown = nullptr;
    for (const auto& e : edits)
        if (e.time >= 0) {
            shown = &e;
            break;
        }
    if (!shown) {
        if (!edits.empty())
            warnings.push_back("the video track's edit list shows no media; every sample is presented");
        return {0, durations.size()};
    }
    if (shown->rate != 0x10000)
        warnings.push_back("the video track's edit plays at rate " + decimal(double(shown->rate) / 65536.0) +
                           "; frames are read at normal speed");
    // Compare in the media timescale scaled by the movie's, exactly.
    using u128 = unsigned __int128;
    const u128 start = u128(uint64_t(shown->time)) * movie_timescale;
    u128 end;
    if (shown->duration == 0) {
        end = ~u128(0);
    } else {
        MOV_ENSURE(movie_timescale != 0, "the movie's timescale is 0");
        end = start + u128(shown->duration) * timescale;
    }
    u128 time = 0;
    size_t first = durations.size(), last = durations.size();
    for (size_t i = 0; i < durations.size(); i++) {
        if (time >= end) {
            last = i;
            break;
        }
        if (time >= start && first == durations.size()) first = i;
        time += u128(durations[i]) * movie_timescale;
    }
    return {first, std::max(last, first)};
}

// An enabled video track's media, before its sample table is resolved.
struct Video {
    uint8_t fourcc[4];
    uint32_t timescale;
    Span tkhd;
    std::optional<Span> elst;
    std::vector<Atom> stbl;

    const Atom* table(const char* kind) const { return find(stbl, kind); }

    // Each sample's size, from `stsz` or `stz2` (src/mov.rs:385-419).
    std::vector<uint32_t> sizes() const {
        if (const Atom* a = table("stsz")) {
            const uint32_t size = u32_at(a->body, 4, "stsz");
            const size_t count = sample_count(u32_at(a->body, 8, "stsz"));
            if (size != 0) return std::vector<uint32_t>(count, size);
            const Span t = entries(a->body, 12, count, 4, "stsz");
            std::vector<uint32_t> out(count);
            for (size_t i = 0; i < count; i++) out[i] = be32(t.p + 4 * i);
            return out;
        }
        const Atom* a = table("stz2");
        MOV_ENSURE(a, "the video track has no sample sizes (`stsz` or `stz2`)");
        MOV_ENSURE(a->body.n > 7, "truncated `stz2` atom");
        const uint8_t field = a->body.p[7];
        const size_t count = sample_count(u32_at(a->body, 8, "stz2"));
        std::vector<uint32_t> out;
        out.reserve(count);
        if (field == 4) {
            const Span t = entries(a->body, 12, (count + 1) / 2, 1, "stz2");
            for (size_t i = 0; i < count; i++) out.push_back(i & 1 ? (t.p[i / 2] & 15) : (t.p[i / 2] >> 4));
        } else if (field == 8) {
            const Span t = entries(a->body, 12, count, 1, "stz2");
            for (size_t i = 0; i < count; i++) out.push_back(t.p[i]);
        } else if (field == 16) {
            const Span t = entries(a->body, 12, count, 2, "stz2");
            for (size_t i = 0; i < count; i++) out.push_back(uint32_t(t.p[2 * i]) << 8 | t.p[2 * i + 1]);
        } else {
            throw Error("`stz2` field size " + std::to_string(field) + " is not 4, 8 or 16 bits");
        }
        return out;
    }

    // Each sample's duration, from `stts` (src/mov.rs:420-438).
    std::vector<uint32_t> durations(size_t samples) const {
        const Span stts = require(stbl, "stts", "the video track");
        const size_t count = u32_at(stts, 4, "stts");
        const Span t = entries(stts, 8, count, 8, "stts");
        uint64_t total = 0;
        for (size_t i = 0; i < count; i++) total += be32(t.p + 8 * i);
        MOV_ENSURE(total == samples, "the video track's sample table disagrees: `stts` times " +
                                         std::to_string(total) + " samples, the sizes list " +
                                         std::to_string(samples));
        std::vector<uint32_t> out;
        out.reserve(samples);
        for (size_t i = 0; i < count; i++) {
            const uint32_t duration = be32(t.p + 8 * i + 4);
            MOV_ENSURE(duration > 0, "the video track has a sample of duration 0");
            out.insert(out.end(), be32(t.p + 8 * i), duration);
        }
        return out;
    }

    // Each sample's place in the file, from the chunk offsets and `stsc`
    // (src/mov.rs:439-505).
    std::vector<Sample> locate(const std::vector<uint32_t>& sizes, uint64_t length) const {
        std::vector<uint64_t> chunks;
        if (const Atom* a = table("stco")) {
            const size_t count = u32_at(a->body, 4, "stco");
            const Span t = entries(a->body, 8, count, 4, "stco");
            for (size_t i = 0; i < count; i++) chunks.push_back(be32(t.p + 4 * i));
        } else {
            const Atom* b = table("co64");
            MOV_ENSURE(b, "the video track has no chunk offsets (`stco` or `co64`)");
            const size_t count = u32_at(b->body, 4, "co64");
            const Span t = entries(b->body, 8, count, 8, "co64");
            for (size_t i = 0; i < count; i++) chunks.push_back(be64(t.p + 8 * i));
        }
        const Span stsc = require(stbl, "stsc", "the video track");
        const size_t count = u32_at(stsc, 4, "stsc");
        const Span t = entries(stsc, 8, count, 12, "stsc");
        std::vector<std::pair<size_t, size_t>> runs;
        for (size_t i = 0; i < count; i++) runs.emplace_back(be32(t.p + 12 * i), be32(t.p + 12 * i + 4));
        bool ordered = !runs.empty() && runs.front().first == 1 && runs.back().first <= chunks.size();
        for (size_t i = 1; ordered && i < runs.size(); i++) ordered = runs[i - 1].first < runs[i].first;
        MOV_ENSURE(ordered, "the video track's `stsc` does not list runs of its " + std::to_string(chunks.size()) +
                                " chunks from chunk 1 in order");
        std::vector<Sample> samples;
        samples.reserve(sizes.size());
        size_t next_size = 0;
        for (size_t i = 0; i < runs.size(); i++) {
            const size_t first = runs[i].first, per_chunk = runs[i].second;
            const size_t end = i + 1 < runs.size() ? runs[i + 1].first - 1 : chunks.size();
            for (size_t c = first - 1; c < end; c++) {
                uint64_t offset = chunks[c];
                for (size_t k = 0; k < per_chunk; k++) {
                    MOV_ENSURE(next_size < sizes.size(),
                               "the video track's sample table disagrees: its chunks hold more than the " +
                                   std::to_string(sizes.size()) + " samples it sizes");
                    const uint32_t size = sizes[next_size++];
                    const uint64_t stop = offset > UINT64_MAX - size ? UINT64_MAX : offset + size;
                    MOV_ENSURE(stop <= length, "sample " + std::to_string(samples.size()) + " (bytes " +
                                                   std::to_string(offset) + ".." + std::to_string(stop) +
                                                   ") lies beyond the end of the file at " + std::to_string(length) +
                                                   " bytes (a truncated file?)");
                    samples.push_back({offset, size});
                    offset = stop;
                }
            }
        }
        MOV_ENSURE(samples.size() == sizes.size(), "the video track's sample table disagrees: its chunks hold " +
                                                       std::to_string(samples.size()) + " of the " +
                                                       std::to_string(sizes.size()) + " samples it sizes");
        return samples;
    }

    Track read(uint64_t length, uint32_t movie_timescale) const {
        const auto sz = sizes();
        MOV_ENSURE(!sz.empty(), "the video track has no samples");
        const auto du = durations(sz.size());
        const auto samples = locate(sz, length);
        const auto [mode, variable] = common_duration(du);
        const uint32_t divisor = gcd(timescale, mode);
        Track t;
        std::memcpy(t.fourcc, fourcc, 4);
        t.orientation = orientation(tkhd, t.warnings);
        std::pair<size_t, size_t> presented{0, samples.size()};
        if (elst) presented = edit(*elst, du, timescale, movie_timescale, t.warnings);
        MOV_ENSURE(presented.first < presented.second, "the video track's edit list presents none of its " +
                                                           std::to_string(samples.size()) + " samples");
        t.fps_num = timescale / divisor;
        t.fps_den = mode / divisor;
        t.variable_durations = variable;
        t.samples.assign(samples.begin() + presented.first, samples.begin() + presented.second);
        return t;
    }
};

// `trak`'s media when it is an enabled video track (src/mov.rs:303-341).
std::optional<Video> video_track(Span trak) {
    const auto atoms = children(trak);
    const Span tkhd = require(atoms, "tkhd", "a track");
    if ((u32_at(tkhd, 0, "tkhd") & 1) == 0) return std::nullopt;
    const auto mdia = children(require(atoms, "mdia", "a track"));
    // Version and flags, component type, then the subtype.
    const uint32_t handler = u32_at(require(mdia, "hdlr", "a track's media"), 8, "hdlr");
    if (handler != be32(reinterpret_cast<const uint8_t*>("vide"))) return std::nullopt;
    const uint32_t timescale = times(require(mdia, "mdhd", "the video track"), "mdhd").second;
    MOV_ENSURE(timescale > 0, "the video track's timescale is 0");
    const auto minf = children(require(mdia, "minf", "the video track"));
    Video v;
    v.stbl = children(require(minf, "stbl", "the video track"));
    const Span stsd = require(v.stbl, "stsd", "the video track");
    MOV_ENSURE(u32_at(stsd, 4, "stsd") > 0, "the video track has no sample description");
    // Version and flags, entry count, then the first entry's size and fourcc.
    const uint32_t fc = u32_at(stsd, 12, "stsd");
    for (int i = 0; i < 4; i++) v.fourcc[i] = uint8_t(fc >> (24 - 8 * i));
    v.timescale = timescale;
    v.tkhd = tkhd;
    if (const Atom* edts = find(atoms, "edts"))
        for (const Atom& a : children(edts->body))
            if (a.is("elst")) {
                v.elst = a.body;
                break;
            }
    return v;
}

Track parse_movie(Span moov, uint64_t length, prr_mov_accept_fn accept, void* user) {
    const auto atoms = children(moov);
    const auto [creation_time, movie_timescale] = times(require(atoms, "mvhd", "the movie"), "mvhd");
    std::optional<std::string> rejected;
    for (const Atom& a : atoms) {
        if (!a.is("trak")) continue;
        auto video = video_track(a.body);
        if (!video) continue;
        if (!accept(video->fourcc, user)) {
            if (!rejected) rejected = name(video->fourcc);
            continue;
        }
        Track t = video->read(length, movie_timescale);
        if (creation_time != 0) t.creation_time = creation_time;
        if (const Atom* meta = find(atoms, "meta")) {
            // Metadata is optional: a damaged item costs the tags, not the frames.
            try {
                t.metadata = text_metadata(meta->body);
            } catch (const Error& e) {
                t.warnings.push_back(std::string("the movie's metadata is unreadable: ") + e.what());
            }
        }
        return t;
    }
    if (rejected) throw Error("the video track is `" + *rejected + "`, not a format this reader accepts");
    throw Error("the movie has no enabled video track");
}

// An OS error as the crate prints one: the system's text, then the code.
std::string os_error(int code) { return std::string(std::strerror(code)) + " (os error " + std::to_string(code) + ")"; }

// Positional read of `len` bytes at `offset` (src/mov.rs:179-183).
void read_at(int fd, uint64_t offset, uint8_t* buf, size_t len) {
    size_t done = 0;
    while (done < len) {
        const ssize_t r = ::pread(fd, buf + done, len - done, off_t(offset + done));
        if (r < 0 && errno == EINTR) continue;
        if (r <= 0)
            throw Error("reading " + std::to_string(len) + " bytes at byte " + std::to_string(offset) + ": " +
                        (r == 0 ? std::string("failed to fill whole buffer") : os_error(errno)));
        done += size_t(r);
    }
}

// The body of the top-level `moov` atom (src/mov.rs:205-255).
std::vector<uint8_t> read_moov(int fd, uint64_t length) {
    uint64_t position = 0;
    while (position < length) {
        uint8_t header[16] = {};
        const size_t available = size_t(std::min<uint64_t>(length - position, 16));
        MOV_ENSURE(available >= 8, "truncated atom header at byte " + std::to_string(position));
        read_at(fd, position, header, available);
        const uint8_t* kind = header + 4;
        bool first = false;
        for (const char* k : kFirstAtoms) first |= std::memcmp(kind, k, 4) == 0;
        MOV_ENSURE(position > 0 || first, "not a QuickTime movie: it starts with `" + name(kind) +
                                              "`, not `ftyp` or `moov`");
        uint64_t header_size, size;
        const uint32_t s32 = be32(header);
        if (s32 == 1) {
            MOV_ENSURE(available == 16, "truncated `" + name(kind) + "` atom header");
            header_size = 16;
            size = be64(header + 8);
        } else if (s32 == 0) {
            header_size = 8;
            size = length - position;
        } else {
            header_size = 8;
            size = s32;
        }
        MOV_ENSURE(size >= header_size, "invalid `" + name(kind) + "` atom size " + std::to_string(size) +
                                            " at byte " + std::to_string(position));
        MOV_ENSURE(size <= length - position, "truncated `" + name(kind) + "` atom at byte " +
                                                  std::to_string(position) + ": it claims " + std::to_string(size) +
                                                  " bytes and the file has " + std::to_string(length - position) +
                                                  " left (an interrupted recording?)");
        if (std::memcmp(kind, "moov", 4) == 0) {
            const uint64_t body = size - header_size;
            MOV_ENSURE(body <= kMaxMoov, "the `moov` atom is " + std::to_string(body) + " bytes, more than the " +
                                             std::to_string(kMaxMoov) + " this reader accepts");
            std::vector<uint8_t> moov(static_cast<size_t>(body));
            read_at(fd, position + header_size, moov.data(), moov.size());
            return moov;
        }
        position += size;
    }
    if (length == 0) throw Error("not a QuickTime movie: the file is empty");
    throw Error("the movie has no `moov` atom, so its frames cannot be found (an interrupted recording?)");
}

// is_prores_raw_fourcc (src/lib.rs:68-75): `aprn` or `aprh`, any case.
int prores_raw(const uint8_t* fourcc, void*) {
    char lower[4];
    for (int i = 0; i < 4; i++) lower[i] = char(fourcc[i] >= 'A' && fourcc[i] <= 'Z' ? fourcc[i] + 32 : fourcc[i]);
    return std::memcmp(lower, "aprn", 4) == 0 || std::memcmp(lower, "aprh", 4) == 0;
}

void put_message(char* out, size_t cap, const std::string& m) {
    if (!out || cap == 0) return;
    const size_t n = std::min(cap - 1, m.size());
    std::memcpy(out, m.data(), n);
    out[n] = '\0';
}

}  // namespace
}  // namespace mov
}  // namespace prr

struct prr_mov_track {
    int fd = -1;
    prr::mov::Track track;
};

namespace prr {
// For the clip pipeline: positional reads with the crate's messages, on a
// track's file or on any descriptor.
int mov_read_fd(int fd, uint64_t offset, uint8_t* buf, size_t len, char* message, size_t message_cap) {
    try {
        mov::read_at(fd, offset, buf, len);
        return PRR_OK;
    } catch (const mov::Error& e) {
        mov::put_message(message, message_cap, e.what());
        return PRR_ERR_MOVIE;
    }
}
int mov_track_fd(const prr_mov_track* t) { return t ? t->fd : -1; }
}  // namespace prr

using namespace prr::mov;

extern "C" {

int prr_mov_open(const char* path, prr_mov_accept_fn accept, void* user, prr_mov_track** out, char* message,
                 size_t message_cap) {
    if (!path || !out) return PRR_ERR_INVALID;
    *out = nullptr;
    const int fd = ::open(path, O_RDONLY | O_CLOEXEC);
    if (fd < 0) {
        put_message(message, message_cap, os_error(errno));
        return PRR_ERR_MOVIE;
    }
    try {
        struct stat st;
        if (::fstat(fd, &st) != 0)
            throw Error("reading the file's length: " + os_error(errno));
        const uint64_t length = uint64_t(st.st_size);
        const auto moov = read_moov(fd, length);
        auto* t = new prr_mov_track;
        t->fd = fd;
        try {
            t->track = parse_movie(Span{moov.data(), moov.size()}, length, accept ? accept : prores_raw, user);
        } catch (...) {
            delete t;
            throw;
        }
        *out = t;
        put_message(message, message_cap, "");
        return PRR_OK;
    } catch (const Error& e) {
        ::close(fd);
        put_message(message, message_cap, e.what());
        return PRR_ERR_MOVIE;
    } catch (const std::bad_alloc&) {
        ::close(fd);
        put_message(message, message_cap, "out of memory");
        return PRR_ERR_NO_MEMORY;
    }
}

void prr_mov_close(prr_mov_track* t) {
    if (!t) return;
    if (t->fd >= 0) ::close(t->fd);
    delete t;
}

int prr_mov_get_info(const prr_mov_track* t, prr_mov_info* info) {
    if (!t || !info) return PRR_ERR_INVALID;
    std::memset(info, 0, sizeof(*info));
    std::memcpy(info->fourcc, t->track.fourcc, 4);
    info->fps_num = t->track.fps_num;
    info->fps_den = t->track.fps_den;
    info->variable_durations = t->track.variable_durations ? 1 : 0;
    info->orientation = uint8_t(t->track.orientation);
    info->has_creation_time = t->track.creation_time ? 1 : 0;
    info->creation_time = t->track.creation_time.value_or(0);
    info->n_samples = t->track.samples.size();
    info->n_warnings = uint32_t(t->track.warnings.size());
    info->n_metadata = uint32_t(t->track.metadata.size());
    return PRR_OK;
}

int prr_mov_get_samples(const prr_mov_track* t, size_t first, size_t count, prr_mov_sample* out) {
    if (!t || (!out && count > 0)) return PRR_ERR_INVALID;
    if (first > t->track.samples.size() || count > t->track.samples.size() - first) return PRR_ERR_INVALID;
    for (size_t i = 0; i < count; i++) {
        out[i].offset = t->track.samples[first + i].offset;
        out[i].size = t->track.samples[first + i].size;
        out[i].pad = 0;
    }
    return PRR_OK;
}

const char* prr_mov_warning(const prr_mov_track* t, size_t i) {
    if (!t || i >= t->track.warnings.size()) return nullptr;
    return t->track.warnings[i].c_str();
}

int prr_mov_metadata(const prr_mov_track* t, size_t i, const char** key, const char** value) {
    if (!t || !key || !value || i >= t->track.metadata.size()) return PRR_ERR_INVALID;
    *key = t->track.metadata[i].first.c_str();
    *value = t->track.metadata[i].second.c_str();
    return PRR_OK;
}

int prr_mov_read_at(const prr_mov_track* t, uint64_t offset, uint8_t* buf, size_t len, char* message,
                    size_t message_cap) {
    if (!t || (!buf && len > 0)) return PRR_ERR_INVALID;
    return prr::mov_read_fd(t->fd, offset, buf, len, message, message_cap);
}

}  // extern "C"
