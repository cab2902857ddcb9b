// sg_oracle.cpp -- CPU reference of the learned demosaic surrogate (test
// infrastructure; the network is stated in sg_oracle.h).

#include "sg_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace {

constexpr int kIn = 16, kHidden = 32, kHead = 16, kLayers = 7;
constexpr int cin_of(int l) { return l == 0 ? kIn : kHidden; }
constexpr int cout_of(int l) { return l == kLayers - 1 ? kHead : kHidden; }

size_t layer_offset(int l) {
    size_t off = 0;
    for (int k = 0; k < l; k++) off += size_t(cout_of(k)) * cin_of(k) * 9 + cout_of(k);
    return off;
}

// Round to the nearest bf16, ties to even (as __float2bfloat16_rn).
float bf16(float v) {
    uint32_t u;
    std::memcpy(&u, &v, 4);
    if ((u & 0x7F800000u) == 0x7F800000u) {  // inf / nan: keep (quiet nan)
        if (u & 0x7FFFFFu) u |= 0x400000u;
        u &= 0xFFFF0000u;
    } else {
        const uint32_t lsb = (u >> 16) & 1u;
        u += 0x7FFFu + lsb;
        u &= 0xFFFF0000u;
    }
    float r;
    std::memcpy(&r, &u, 4);
    return r;
}

// One 3x3 convolution, zero padding: out[co][y][x] = b[co] + sum w * in.
void conv(const float* in, int cin, int h, int w, const float* wt, const float* bias, int cout, bool rnd,
          float* out) {
    std::vector<float> wr(size_t(cout) * cin * 9);
    for (size_t i = 0; i < wr.size(); i++) wr[i] = rnd ? bf16(wt[i]) : wt[i];
    for (int co = 0; co < cout; co++)
        for (int y = 0; y < h; y++)
            for (int x = 0; x < w; x++) {
                float acc = bias[co];
                for (int ci = 0; ci < cin; ci++)
                    for (int t = 0; t < 9; t++) {
                        const int yy = y + t / 3 - 1, xx = x + t % 3 - 1;
                        if (yy < 0 || yy >= h || xx < 0 || xx >= w) continue;
                        acc += wr[(size_t(co) * cin + ci) * 9 + t] * in[(size_t(ci) * h + yy) * w + xx];
                    }
                out[(size_t(co) * h + y) * w + x] = acc;
            }
}

inline float variance(float v, float off, const float* n) {  // demosaic.rs:423-426
    const float t = off + v;
    return n[2] + std::max(n[1], n[0] * (t * t));
}

}  // namespace

extern "C" {

size_t orc_sg_param_count(void) { return layer_offset(kLayers); }

int orc_sg_pack(const orc_header* hdr, const uint16_t* samples, const orc_params* p, float* in16,
                float* base3) {
    const int w = hdr->width, h = hdr->height;
    const int stride = (w + 15) & ~15;
    const int wq = (w + 1) / 2, hq = (h + 1) / 2;
    const int rr = p->cfa_phase >> 1, rc = p->cfa_phase & 1;
    const float bs = float(p->black) * p->one_over_range;
    auto nrm = [&](int x, int y) {
        x = std::min(x, w - 1);
        y = std::min(y, h - 1);
        const uint16_t lin = orc_curve_linearize(hdr->curve, samples[size_t(y) * stride + x]);
        return p->one_over_range * float(int32_t(lin) - p->black);
    };
    const size_t plane = size_t(wq) * hq;
    // Mean green of quad (i, j), coordinates clamped to the quad grid.
    auto green = [&](int i, int j) {
        i = std::clamp(i, 0, wq - 1);
        j = std::clamp(j, 0, hq - 1);
        const float gr = nrm(2 * i + 1 - rc, 2 * j + rr);
        const float gb = nrm(2 * i + rc, 2 * j + 1 - rr);
        return (gr + gb) * 0.5f;
    };
    // Network quad (i, j) is picture quad (si, sj): mirrored by the red
    // sensel's column and row, so that every pattern is seen as RGGB.
    const int ex = rc ? -1 : 1, sy = rr ? -1 : 1;
    for (int j = 0; j < hq; j++)
        for (int i = 0; i < wq; i++) {
            const int si = rc ? wq - 1 - i : i, sj = rr ? hq - 1 - j : j;
            const int x0 = 2 * si, y0 = 2 * sj;
            const float r = nrm(x0 + rc, y0 + rr) * p->wb[0];
            const float gr = nrm(x0 + 1 - rc, y0 + rr);
            const float gb = nrm(x0 + rc, y0 + 1 - rr);
            const float b = nrm(x0 + 1 - rc, y0 + 1 - rr) * p->wb[1];
            const float gm = (gr + gb) * 0.5f;
            const float noise = 64.0f * std::sqrt(variance(gm, bs, p->noise));
            const float ge = green(si + ex, sj), gw = green(si - ex, sj), gs = green(si, sj + sy),
                        gn = green(si, sj - sy);
            const float gx = (ge - gw) * 0.5f, gy = (gs - gn) * 0.5f;
            const float lap = gm - ((ge + gw) + (gs + gn)) * 0.25f;
            const size_t q = size_t(j) * wq + i;
            const float v[9] = {(r - gm) * 4.0f, (gr - gm) * 4.0f, (gb - gm) * 4.0f, (b - gm) * 4.0f, noise,
                                gm, gx * 4.0f, gy * 4.0f, lap * 4.0f};
            for (int c = 0; c < kIn; c++) in16[c * plane + q] = c < 9 ? bf16(v[c]) : 0.0f;
            base3[q] = r;
            base3[plane + q] = gm;
            base3[2 * plane + q] = b;
        }
    return ORC_OK;
}

void orc_sg_forward(const float* in16, int h, int w, const float* params, int round_bf16, float* acts,
                    float* head) {
    const size_t plane = size_t(h) * w;
    std::vector<float> a(kIn * plane), b(kHidden * plane);
    for (size_t i = 0; i < a.size(); i++) a[i] = round_bf16 ? bf16(in16[i]) : in16[i];
    for (int l = 0; l < kLayers; l++) {
        const float* wt = params + layer_offset(l);
        const float* bias = wt + size_t(cout_of(l)) * cin_of(l) * 9;
        if (l == kLayers - 1) {
            conv(a.data(), cin_of(l), h, w, wt, bias, kHead, round_bf16 != 0, head);
            break;
        }
        b.assign(kHidden * plane, 0.0f);
        conv(a.data(), cin_of(l), h, w, wt, bias, kHidden, round_bf16 != 0, b.data());
        for (auto& v : b) {
            v = std::max(v, 0.0f);
            if (round_bf16) v = bf16(v);
        }
        if (acts) std::memcpy(acts + size_t(l) * kHidden * plane, b.data(), b.size() * 4);
        a.swap(b);
    }
}

void orc_sg_output(const float* head, const float* base3, int hq, int wq, int width, int height, int cfa,
                   const float* m9, float* r, float* g, float* b) {
    const size_t plane = size_t(hq) * wq;
    const int rr = cfa >> 1, rc = cfa & 1;
    for (int y = 0; y < height; y++)
        for (int x = 0; x < width; x++) {
            const int qi = rc ? wq - 1 - (x >> 1) : (x >> 1), qj = rr ? hq - 1 - (y >> 1) : (y >> 1);
            const size_t q = size_t(qj) * wq + qi;
            const int s = ((y & 1) ^ rr) * 2 + ((x & 1) ^ rc);
            float rv = std::min(head[(0 + s) * plane + q] + base3[q], 1.0f);
            float gv = std::min(head[(4 + s) * plane + q] + base3[plane + q], 1.0f);
            float bv = std::min(head[(8 + s) * plane + q] + base3[2 * plane + q], 1.0f);
            if (m9) {
                const float r0 = rv, g0 = gv, b0 = bv;
                rv = std::fma(b0, m9[2], std::fma(r0, m9[0], g0 * m9[1]));
                gv = std::fma(b0, m9[5], std::fma(r0, m9[3], g0 * m9[4]));
                bv = std::fma(b0, m9[8], std::fma(r0, m9[6], g0 * m9[7]));
            }
            const size_t o = size_t(y) * width + x;
            r[o] = rv;
            g[o] = gv;
            b[o] = bv;
        }
}

double orc_sg_loss(const float* head, const float* base3, int hq, int wq, int width, int height,
                   const float* tr, const float* tg, const float* tb, float* dhead) {
    const size_t plane = size_t(hq) * wq;
    std::memset(dhead, 0, kHead * plane * sizeof(float));
    const double n = 3.0 * double(width) * double(height);
    double loss = 0.0;
    const float* t[3] = {tr, tg, tb};
    for (int y = 0; y < height; y++)
        for (int x = 0; x < width; x++) {
            const size_t q = size_t(y >> 1) * wq + (x >> 1);
            const int s = (y & 1) * 2 + (x & 1);
            for (int c = 0; c < 3; c++) {
                const float out = head[(c * 4 + s) * plane + q] + base3[c * plane + q];
                const float d = out - t[c][size_t(y) * width + x];
                loss += double(d) * d;
                dhead[(c * 4 + s) * plane + q] = float(2.0 * d / n);
            }
        }
    return loss / n;
}

void orc_sg_backward(const float* in16, int h, int w, const float* params, const float* acts,
                     const float* dhead, float* dparams) {
    const size_t plane = size_t(h) * w;
    std::memset(dparams, 0, orc_sg_param_count() * sizeof(float));
    std::vector<float> dy(dhead, dhead + kHead * plane), dx;
    for (int l = kLayers - 1; l >= 0; l--) {
        const int cin = cin_of(l), cout = cout_of(l);
        const float* wt = params + layer_offset(l);
        float* dw = dparams + layer_offset(l);
        float* db = dw + size_t(cout) * cin * 9;
        const float* x = l == 0 ? in16 : acts + size_t(l - 1) * kHidden * plane;
        for (int co = 0; co < cout; co++)
            for (size_t p = 0; p < plane; p++) db[co] += dy[co * plane + p];
        for (int co = 0; co < cout; co++)
            for (int ci = 0; ci < cin; ci++)
                for (int t = 0; t < 9; t++) {
                    double acc = 0.0;
                    for (int yy = 0; yy < h; yy++)
                        for (int xx = 0; xx < w; xx++) {
                            const int sy = yy + t / 3 - 1, sx = xx + t % 3 - 1;
                            if (sy < 0 || sy >= h || sx < 0 || sx >= w) continue;
                            acc += double(dy[co * plane + size_t(yy) * w + xx]) * x[ci * plane + size_t(sy) * w + sx];
                        }
                    dw[(size_t(co) * cin + ci) * 9 + t] = float(acc);
                }
        if (l == 0) break;
        // Gradient of the previous activation, through its ReLU.
        dx.assign(size_t(cin) * plane, 0.0f);
        for (int ci = 0; ci < cin; ci++)
            for (int yy = 0; yy < h; yy++)
                for (int xx = 0; xx < w; xx++) {
                    float acc = 0.0f;
                    for (int co = 0; co < cout; co++)
                        for (int t = 0; t < 9; t++) {
                            const int oy = yy - (t / 3 - 1), ox = xx - (t % 3 - 1);
                            if (oy < 0 || oy >= h || ox < 0 || ox >= w) continue;
                            acc += wt[(size_t(co) * cin + ci) * 9 + t] * dy[co * plane + size_t(oy) * w + ox];
                        }
                    const size_t i = ci * plane + size_t(yy) * w + xx;
                    dx[i] = x[i] > 0.0f ? acc : 0.0f;
                }
        dy.swap(dx);
    }
}

}  // extern "C"
