// develop.cu -- linearization and the raw conversion (demosaic, white
// balance, output matrix) on sm_100a.
//
// k_develop fuses the crate's three passes (src/demosaic.rs:356-398) into one
// kernel over 32x32 output tiles:
//  1. normalized values (curve folded with (v - black) / range,
//     src/demosaic.rs:293-298) of the tile plus a 3-sensel halo, loaded with
//     the picture-edge clamping the passes use, into shared memory;
//  2. the green pass (src/demosaic.rs:481-541) over the tile plus a 1-sensel
//     halo, keeping in shared memory the (red or blue, green) pair of every
//     sensel and the per-sensel noise terms the chroma pass needs (variance
//     and its square root), each computed once instead of once per use;
//  3. the chroma pass (src/demosaic.rs:572-688) and the matrix
//     (src/demosaic.rs:700-720) per 2x2 Bayer quad, so a thread's work does
//     not depend on its column parity, with 8-byte coalesced stores.
// Every operation is an IEEE round-to-nearest intrinsic, with fused
// multiply-adds exactly where the crate calls mul_add, so the output is bit
// for bit the crate's.

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstring>

#include "device_common.cuh"
#include "fastdiv.cuh"
#include "kernels.h"

namespace prr {

namespace {

__device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float dv(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ float rt(float a) { return __fsqrt_rn(a); }
__device__ __forceinline__ float fma_(float a, float b, float c) { return __fmaf_rn(a, b, c); }

struct Noise {
    float a, b, c;
};

// variance, src/demosaic.rs:423-426.
__device__ __forceinline__ float variance(float v, float off, const Noise& n) {
    const float t = add(off, v);
    return add(n.c, fmaxf(n.b, mul(n.a, mul(t, t))));
}

// dot4, src/demosaic.rs:431-433.
__device__ __forceinline__ float dot4(float a0, float a1, float a2, float a3, float b0, float b1,
                                      float b2, float b3) {
    return fma_(a3, b3, fma_(a2, b2, fma_(a0, b0, mul(a1, b1))));
}

// mirror, src/demosaic.rs:547-557.
__device__ __forceinline__ void mirror(float* d, int pos, int len, float c) {
    if (pos == 0) {
        d[0] = d[1];
        d[2] = d[3];
    } else if (pos == 1) {
        d[2] = c;
    } else if (pos == len - 1) {
        d[1] = d[0];
        d[3] = d[2];
    } else if (pos == len - 2) {
        d[3] = c;
    }
}

// estimate, src/demosaic.rs:572-604, with the per-sensel terms precomputed:
// var_x = variance(x), sx = sqrt(var_x), sg = sqrt(variance(g)).
__device__ __forceinline__ float estimate(const float* xx, const float* gg, const float* var_x,
                                          const float* sx, const float* sg, float cg, float cs) {
    const float mean_x = dot4(xx[0], xx[1], xx[2], xx[3], 0.25f, 0.25f, 0.25f, 0.25f);
    // Also falls back when the comparison is unordered (NaN).
    if (!(cs < cg)) return mean_x;
    bool above = true;
#pragma unroll
    for (int i = 0; i < 4; i++) above &= (sx[i] < xx[i]) & (sg[i] < gg[i]);
    if (!above) return mean_x;
    float lo[4], mid[4], hi[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        lo[i] = dv(mul(sub(cg, cs), sub(xx[i], sx[i])), add(sg[i], gg[i]));
        mid[i] = dv(mul(cg, xx[i]), gg[i]);
        hi[i] = dv(mul(add(cs, cg), add(sx[i], xx[i])), sub(gg[i], sg[i]));
    }
    const float spread = dot4(sub(mid[0], lo[0]), sub(mid[1], lo[1]), sub(mid[2], lo[2]), sub(mid[3], lo[3]),
                              sub(hi[0], mid[0]), sub(hi[1], mid[1]), sub(hi[2], mid[2]), sub(hi[3], mid[3]));
    const float mean_mid = dot4(mid[0], mid[1], mid[2], mid[3], 0.25f, 0.25f, 0.25f, 0.25f);
    const float dm0 = sub(mid[0], mean_mid), dm1 = sub(mid[1], mean_mid), dm2 = sub(mid[2], mean_mid),
                dm3 = sub(mid[3], mean_mid);
    const float b = fma_(spread, 0.75f, dot4(dm0, dm1, dm2, dm3, dm0, dm1, dm2, dm3));
    const float dx0 = sub(xx[0], mean_x), dx1 = sub(xx[1], mean_x), dx2 = sub(xx[2], mean_x),
                dx3 = sub(xx[3], mean_x);
    const float vsum = dot4(var_x[0], var_x[1], var_x[2], var_x[3], 1.0f, 1.0f, 1.0f, 1.0f);
    const float a = fma_(vsum, 0.75f, dot4(dx0, dx1, dx2, dx3, dx0, dx1, dx2, dx3));
    const float weight = dv(a, add(b, a));
    return fma_(sub(mean_mid, mean_x), weight, mean_x);
}

// estimate() with lanes (u, v, u, v): two opposite neighbours each counted
// twice (src/demosaic.rs:674-678). Each distinct lane is computed once; the
// sums keep the four-lane order of dot4, so the result is estimate()'s.
__device__ __forceinline__ float estimate2(float xu, float xv, float gu, float gv, float vu, float vv,
                                           float su, float sv, float tu, float tv, float cg, float cs) {
    const float mean_x = fma_(xv, 0.25f, fma_(xu, 0.25f, fma_(xu, 0.25f, mul(xv, 0.25f))));
    if (!(cs < cg)) return mean_x;
    if (!((su < xu) & (tu < gu) & (sv < xv) & (tv < gv))) return mean_x;
    const float lo_u = dv(mul(sub(cg, cs), sub(xu, su)), add(tu, gu));
    const float lo_v = dv(mul(sub(cg, cs), sub(xv, sv)), add(tv, gv));
    const float mid_u = dv(mul(cg, xu), gu);
    const float mid_v = dv(mul(cg, xv), gv);
    const float hi_u = dv(mul(add(cs, cg), add(su, xu)), sub(gu, tu));
    const float hi_v = dv(mul(add(cs, cg), add(sv, xv)), sub(gv, tv));
    const float ml_u = sub(mid_u, lo_u), ml_v = sub(mid_v, lo_v);
    const float hm_u = sub(hi_u, mid_u), hm_v = sub(hi_v, mid_v);
    const float spread = fma_(ml_v, hm_v, fma_(ml_u, hm_u, fma_(ml_u, hm_u, mul(ml_v, hm_v))));
    const float mean_mid = fma_(mid_v, 0.25f, fma_(mid_u, 0.25f, fma_(mid_u, 0.25f, mul(mid_v, 0.25f))));
    const float dm_u = sub(mid_u, mean_mid), dm_v = sub(mid_v, mean_mid);
    const float b = fma_(spread, 0.75f, fma_(dm_v, dm_v, fma_(dm_u, dm_u, fma_(dm_u, dm_u, mul(dm_v, dm_v)))));
    const float dx_u = sub(xu, mean_x), dx_v = sub(xv, mean_x);
    const float vsum = fma_(vv, 1.0f, fma_(vu, 1.0f, fma_(vu, 1.0f, mul(vv, 1.0f))));
    const float a = fma_(vsum, 0.75f, fma_(dx_v, dx_v, fma_(dx_u, dx_u, fma_(dx_u, dx_u, mul(dx_v, dx_v)))));
    const float weight = dv(a, add(b, a));
    return fma_(sub(mean_mid, mean_x), weight, mean_x);
}

// Packed pairs of f32 (sm_100 f32x2 arithmetic): each lane is rounded as the
// scalar operation rounds it, so two sites computed as the lanes of one pair
// give the scalar results bit for bit in half the issued instructions.
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) {
    unsigned long long x, y, r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(x) : "f"(a.x), "f"(a.y));
    asm("mov.b64 %0, {%1, %2};" : "=l"(y) : "f"(b.x), "f"(b.y));
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(x), "l"(y));
    float2 o;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(o.x), "=f"(o.y) : "l"(r));
    return o;
}
__device__ __forceinline__ float2 bc(float v) { return make_float2(v, v); }
__device__ __forceinline__ float2 dot4x2(float2 a0, float2 a1, float2 a2, float2 a3, float2 b0, float2 b1, float2 b2,
                                         float2 b3) {
    return fma2(a3, b3, fma2(a2, b2, fma2(a0, b0, mul2(a1, b1))));
}
// variance() of two values, one a lane.
__device__ __forceinline__ float2 variance2(float2 v, float off, const Noise& n) {
    const float2 t = add2(bc(off), v);
    const float2 m = mul2(bc(n.a), mul2(t, t));
    return add2(bc(n.c), make_float2(fmaxf(n.b, m.x), fmaxf(n.b, m.y)));
}

// The estimates' last quotient, weight = a / (b + a), of both lanes. Its
// numerator a is at least three times the noise floor; its denominator
// grows with the spread of the estimate's ratios and, for extreme
// neighbourhoods, can leave the range the paired division is exact in, so
// lanes whose denominator is above 2^60 take div.rn.
template <bool FAST>
__device__ __forceinline__ float2 weight_x2(float2 a, float2 den, bool okx, bool oky) {
    float2 weight = a;
    if (FAST && !((okx & !(den.x <= 0x1p60f)) | (oky & !(den.y <= 0x1p60f)))) {
        weight = div_rn_x2(a, den);
    } else {
        if (okx) weight.x = dv(a.x, den.x);
        if (oky) weight.y = dv(a.y, den.y);
    }
    return weight;
}

// estimate() of two sites, one a lane (src/demosaic.rs:572-604). A lane
// whose test fails returns its mean. FAST: the quotients by the paired
// division (fastdiv.cuh), both lanes at once; else a failing lane's
// divisions are skipped.
template <bool FAST>
__device__ __forceinline__ float2 estimate_x2(const float2* xx, const float2* gg, const float2* var_x,
                                              const float2* sx, const float2* sg, float2 cg, float2 cs) {
    const float2 q = bc(0.25f);
    const float2 mean_x = dot4x2(xx[0], xx[1], xx[2], xx[3], q, q, q, q);
    bool okx = cs.x < cg.x, oky = cs.y < cg.y;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        okx &= (sx[i].x < xx[i].x) & (sg[i].x < gg[i].x);
        oky &= (sx[i].y < xx[i].y) & (sg[i].y < gg[i].y);
    }
    if (!(okx | oky)) return mean_x;
    // The variance and deviation terms first, so that the neighbours'
    // values die as the divisions consume them.
    const float2 dx0 = sub2(xx[0], mean_x), dx1 = sub2(xx[1], mean_x), dx2 = sub2(xx[2], mean_x),
                 dx3 = sub2(xx[3], mean_x);
    // dot4 of the variances with ones: fma(v, 1, s) is add(v, s) exactly.
    const float2 vsum = add2(var_x[3], add2(var_x[2], add2(var_x[0], var_x[1])));
    const float2 a = fma2(vsum, bc(0.75f), dot4x2(dx0, dx1, dx2, dx3, dx0, dx1, dx2, dx3));
    const float2 k1 = sub2(cg, cs), k2 = add2(cs, cg);
    float2 mid[4], ml[4], hm[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const float2 nlo = mul2(k1, sub2(xx[i], sx[i])), dlo = add2(sg[i], gg[i]);
        const float2 nmid = mul2(cg, xx[i]);
        const float2 nhi = mul2(k2, add2(sx[i], xx[i])), dhi = sub2(gg[i], sg[i]);
        float2 lo, md, hi;
        if (FAST) {
            // Both lanes at once (a failing lane's quotients are never used).
            lo = div_rn_x2(nlo, dlo);
            md = div_rn_x2(nmid, gg[i]);
            hi = div_rn_x2(nhi, dhi);
        } else {
            // A failing lane keeps its numerators (never used).
            lo = nlo, md = nmid, hi = nhi;
            if (okx) {
                lo.x = dv(nlo.x, dlo.x);
                md.x = dv(nmid.x, gg[i].x);
                hi.x = dv(nhi.x, dhi.x);
            }
            if (oky) {
                lo.y = dv(nlo.y, dlo.y);
                md.y = dv(nmid.y, gg[i].y);
                hi.y = dv(nhi.y, dhi.y);
            }
        }
        mid[i] = md;
        ml[i] = sub2(md, lo);
        hm[i] = sub2(hi, md);
    }
    const float2 spread = dot4x2(ml[0], ml[1], ml[2], ml[3], hm[0], hm[1], hm[2], hm[3]);
    const float2 mean_mid = dot4x2(mid[0], mid[1], mid[2], mid[3], q, q, q, q);
    const float2 dm0 = sub2(mid[0], mean_mid), dm1 = sub2(mid[1], mean_mid), dm2 = sub2(mid[2], mean_mid),
                 dm3 = sub2(mid[3], mean_mid);
    const float2 b = fma2(spread, bc(0.75f), dot4x2(dm0, dm1, dm2, dm3, dm0, dm1, dm2, dm3));
    const float2 den = add2(b, a);
    const float2 weight = weight_x2<FAST>(a, den, okx, oky);
    const float2 r = fma2(sub2(mean_mid, mean_x), weight, mean_x);
    return make_float2(okx ? r.x : mean_x.x, oky ? r.y : mean_x.y);
}

// estimate2() of two (u, v) neighbour pairs, one a lane.
template <bool FAST>
__device__ __forceinline__ float2 estimate2_x2(float2 xu, float2 xv, float2 gu, float2 gv, float2 vu, float2 vv,
                                               float2 su, float2 sv, float2 tu, float2 tv, float2 cg, float2 cs) {
    const float2 q = bc(0.25f);
    const float2 mean_x = fma2(xv, q, fma2(xu, q, fma2(xu, q, mul2(xv, q))));
    const bool okx = (cs.x < cg.x) & (su.x < xu.x) & (tu.x < gu.x) & (sv.x < xv.x) & (tv.x < gv.x);
    const bool oky = (cs.y < cg.y) & (su.y < xu.y) & (tu.y < gu.y) & (sv.y < xv.y) & (tv.y < gv.y);
    if (!(okx | oky)) return mean_x;
    const float2 dx_u = sub2(xu, mean_x), dx_v = sub2(xv, mean_x);
    const float2 vsum = add2(vv, add2(vu, add2(vu, vv)));
    const float2 a = fma2(vsum, bc(0.75f), fma2(dx_v, dx_v, fma2(dx_u, dx_u, fma2(dx_u, dx_u, mul2(dx_v, dx_v)))));
    const float2 k1 = sub2(cg, cs), k2 = add2(cs, cg);
    const float2 nlo_u = mul2(k1, sub2(xu, su)), nlo_v = mul2(k1, sub2(xv, sv));
    const float2 dlo_u = add2(tu, gu), dlo_v = add2(tv, gv);
    const float2 nmid_u = mul2(cg, xu), nmid_v = mul2(cg, xv);
    const float2 nhi_u = mul2(k2, add2(su, xu)), nhi_v = mul2(k2, add2(sv, xv));
    const float2 dhi_u = sub2(gu, tu), dhi_v = sub2(gv, tv);
    // A failing lane keeps its numerators (never used).
    float2 lo_u = nlo_u, lo_v = nlo_v, mid_u = nmid_u, mid_v = nmid_v, hi_u = nhi_u, hi_v = nhi_v;
    if (FAST) {
        // Both lanes at once (a failing lane's quotients are never used).
        lo_u = div_rn_x2(nlo_u, dlo_u);
        lo_v = div_rn_x2(nlo_v, dlo_v);
        mid_u = div_rn_x2(nmid_u, gu);
        mid_v = div_rn_x2(nmid_v, gv);
        hi_u = div_rn_x2(nhi_u, dhi_u);
        hi_v = div_rn_x2(nhi_v, dhi_v);
    }
    if (!FAST && okx) {
        lo_u.x = dv(nlo_u.x, dlo_u.x);
        lo_v.x = dv(nlo_v.x, dlo_v.x);
        mid_u.x = dv(nmid_u.x, gu.x);
        mid_v.x = dv(nmid_v.x, gv.x);
        hi_u.x = dv(nhi_u.x, dhi_u.x);
        hi_v.x = dv(nhi_v.x, dhi_v.x);
    }
    if (!FAST && oky) {
        lo_u.y = dv(nlo_u.y, dlo_u.y);
        lo_v.y = dv(nlo_v.y, dlo_v.y);
        mid_u.y = dv(nmid_u.y, gu.y);
        mid_v.y = dv(nmid_v.y, gv.y);
        hi_u.y = dv(nhi_u.y, dhi_u.y);
        hi_v.y = dv(nhi_v.y, dhi_v.y);
    }
    const float2 ml_u = sub2(mid_u, lo_u), ml_v = sub2(mid_v, lo_v);
    const float2 hm_u = sub2(hi_u, mid_u), hm_v = sub2(hi_v, mid_v);
    const float2 spread = fma2(ml_v, hm_v, fma2(ml_u, hm_u, fma2(ml_u, hm_u, mul2(ml_v, hm_v))));
    const float2 mean_mid = fma2(mid_v, q, fma2(mid_u, q, fma2(mid_u, q, mul2(mid_v, q))));
    const float2 dm_u = sub2(mid_u, mean_mid), dm_v = sub2(mid_v, mean_mid);
    const float2 b = fma2(spread, bc(0.75f), fma2(dm_v, dm_v, fma2(dm_u, dm_u, fma2(dm_u, dm_u, mul2(dm_v, dm_v)))));
    const float2 den = add2(b, a);
    const float2 weight = weight_x2<FAST>(a, den, okx, oky);
    const float2 r = fma2(sub2(mean_mid, mean_x), weight, mean_x);
    return make_float2(okx ? r.x : mean_x.x, oky ? r.y : mean_x.y);
}

// A tile shape of the develop: TW x TH output sensels (TW a power of two),
// one thread per 2x2 quad. The shapes the autotuner chooses from are
// instantiated below; 32x32 is the default and the only shape a tile mask
// (the learned develop's fallback) addresses.
template <int TW_, int TH_>
struct Tile {
    static constexpr int TW = TW_, TH = TH_;
    static constexpr int NW = TW + 6, NH = TH + 6;  // normalized values, 3-sensel halo
    static constexpr int GW = TW + 2, GH = TH + 2;  // green-pass region, 1-sensel halo
    static constexpr int QW = TW / 2;               // quads per tile row
    static constexpr int kThreads = (TW / 2) * (TH / 2);
    // Resident CTAs per SM the registers are budgeted for (64 a thread).
    static constexpr int kMinBlocks = 1024 / kThreads;
    // The tile's code values with the halo, as one TMA box: NH rows of
    // kBoxW sensels from x0 - 8 (the box's first column must sit on a
    // 16-byte boundary), of which columns kBoxX .. kBoxX + NW - 1 are the
    // ones the tile reads.
    static constexpr int kBoxX = 5;
    static constexpr int kBoxW = (kBoxX + NW + 7) / 8 * 8;
    static_assert((TW & (TW - 1)) == 0 && TW >= 16 && TH % 2 == 0, "tile shape");
};
using Tile32x32 = Tile<32, 32>;
using Tile32x16 = Tile<32, 16>;
using Tile64x16 = Tile<64, 16>;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ bool bar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    return done != 0;
}
// Phase 0 of the tile's barrier, for at most about `limit_ns`.
__device__ __forceinline__ bool bar_wait(uint32_t bar, uint64_t limit_ns) {
    if (bar_try_wait(bar, 0)) return true;
    uint64_t t0;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
    for (uint32_t i = 0; i < (1u << 24); i++) {
        if (bar_try_wait(bar, 0)) return true;
        __nanosleep(64);
        uint64_t t;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
        if (t - t0 > limit_ns) return false;
    }
    return false;
}

template <class T>
struct DevShared {
    static constexpr int NW = T::NW, NH = T::NH, GW = T::GW, GH = T::GH;
    float nrm[NH][NW];
    // Green-pass noise terms of every normalized value once clipped at its
    // own site's limit (1 at green sites, 1/gain at red and blue sites):
    // variance with the green-pass offset, and its square root. The green
    // pass needs them for each neighbour of every red or blue site.
    float gvar[NH][NW];
    float gsd[NH][NW];
    float rb[GH][GW];   // red or blue (0 at green sites)
    float gr[GH][GW];   // green
    float vx[GH][GW];   // variance(rb) with the chroma offset (red/blue sites)
    float sx[GH][GW];   // sqrt(vx)
    float sg[GH][GW];   // sqrt(variance(green)) with the chroma offset
    uint32_t c0[8], cd[8];
};

// White balance, clip and output matrix of a row's two sites as the lanes
// of pairs (src/demosaic.rs:683-720).
__device__ __forceinline__ void finish_x2(float2 r, float2 g, float2 b, const DevelopDesc& d, float2* out) {
    float2 rr = mul2(r, bc(d.wb[0]));
    float2 bb = mul2(b, bc(d.wb[1]));
    rr = make_float2(fminf(rr.x, 1.0f), fminf(rr.y, 1.0f));
    float2 gg = make_float2(fminf(g.x, 1.0f), fminf(g.y, 1.0f));
    bb = make_float2(fminf(bb.x, 1.0f), fminf(bb.y, 1.0f));
    if (d.has_matrix) {
        const float2 m0 = fma2(bb, bc(d.m[2]), fma2(rr, bc(d.m[0]), mul2(gg, bc(d.m[1]))));
        const float2 m1 = fma2(bb, bc(d.m[5]), fma2(rr, bc(d.m[3]), mul2(gg, bc(d.m[4]))));
        const float2 m2 = fma2(bb, bc(d.m[8]), fma2(rr, bc(d.m[6]), mul2(gg, bc(d.m[7]))));
        rr = m0;
        gg = m1;
        bb = m2;
    }
    out[0] = rr;
    out[1] = gg;
    out[2] = bb;
}

// The chroma pass of a quad whose neighbours all lie inside the tile's
// green-pass region and the picture (tiles clear of the edges), every
// neighbour at a fixed offset. A is the column of the quad's red or blue
// site in its first row; the other one sits at (1, 1 - A). The four
// estimates of a quad run two to a pair: the red/blue sites' diagonal
// estimates (src/demosaic.rs:662-669) as the lanes of one pair, each green
// site's horizontal and vertical estimates (src/demosaic.rs:670-680) as the
// lanes of one pair. Returns per quad row the (r, g, b) pairs of its sites.
template <class T, int A, bool FAST>
__device__ __forceinline__ void chroma_quad(const DevShared<T>& S, int gyb, int gxb, bool red0, const DevelopDesc& d,
                                            float2 (&out)[2][3]) {
    constexpr int GW = T::GW;
    // Region site of the quad offset (dy, dx).
    auto idx = [&](int dy, int dx) { return (gyb + dy) * GW + gxb + dx; };
    const float* rb = &S.rb[0][0];
    const float* gr = &S.gr[0][0];
    const float* vx = &S.vx[0][0];
    const float* sx = &S.sx[0][0];
    const float* sg = &S.sg[0][0];
    // The diagonal neighbours, in estimate() order (up-left, down-left,
    // up-right, down-right), of the site (0, A) and of the site (1, 1 - A).
    const int pn[4] = {idx(-1, A - 1), idx(1, A - 1), idx(-1, A + 1), idx(1, A + 1)};
    const int qn[4] = {idx(0, -A), idx(2, -A), idx(0, 2 - A), idx(2, 2 - A)};
    // Two (u, v) neighbour pairs as lanes: lane x (ux, vx_), lane y (uy, vy).
    auto pair2 = [&](int ux, int vx_, int uy, int vy, float2 cg, float2 cs) {
        return estimate2_x2<FAST>(make_float2(rb[ux], rb[uy]), make_float2(rb[vx_], rb[vy]), make_float2(gr[ux], gr[uy]),
                            make_float2(gr[vx_], gr[vy]), make_float2(vx[ux], vx[uy]), make_float2(vx[vx_], vx[vy]),
                            make_float2(sx[ux], sx[uy]), make_float2(sx[vx_], sx[vy]), make_float2(sg[ux], sg[uy]),
                            make_float2(sg[vx_], sg[vy]), cg, cs);
    };
    // Green site (0, 1 - A): lane x its horizontal neighbours qn[0], qn[2],
    // lane y its vertical ones pn[2], pn[3] (A = 0) or pn[0], pn[1] (A = 1).
    const int g0 = idx(0, 1 - A);
    const float gc_0 = gr[g0];
    const float2 e0 = pair2(qn[0], qn[2], pn[A == 0 ? 2 : 0], pn[A == 0 ? 3 : 1], bc(gc_0), bc(sg[g0]));
    // Green site (1, A): horizontal neighbours pn[1], pn[3]; vertical ones
    // qn[0], qn[1] (A = 0) or qn[2], qn[3] (A = 1).
    const int g1 = idx(1, A);
    const float gc_1 = gr[g1];
    const float2 e1 = pair2(pn[1], pn[3], qn[A == 0 ? 0 : 2], qn[A == 0 ? 1 : 3], bc(gc_1), bc(sg[g1]));
    // The red/blue sites' diagonal estimates: lane x the site (0, A), lane y
    // the site (1, 1 - A).
    float2 X[4], G[4], V[4], SX[4], SG[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        X[i] = make_float2(rb[pn[i]], rb[qn[i]]);
        G[i] = make_float2(gr[pn[i]], gr[qn[i]]);
        V[i] = make_float2(vx[pn[i]], vx[qn[i]]);
        SX[i] = make_float2(sx[pn[i]], sx[qn[i]]);
        SG[i] = make_float2(sg[pn[i]], sg[qn[i]]);
    }
    const int ca = idx(0, A), cb = idx(1, 1 - A);
    const float gc_a = gr[ca], gc_b = gr[cb];
    const float2 e = estimate_x2<FAST>(X, G, V, SX, SG, make_float2(gc_a, gc_b), make_float2(sg[ca], sg[cb]));
    const float c_a = rb[ca], c_b = rb[cb];
    // Site (0, A) lies on the first row, (1, 1 - A) on the second; on a red
    // row r is the site's own value, or for a green site the horizontal
    // estimate (src/demosaic.rs:662-688).
    const float r_a = red0 ? c_a : e.x, b_a = red0 ? e.x : c_a;
    const float r_b = red0 ? e.y : c_b, b_b = red0 ? c_b : e.y;
    const float r_g0 = red0 ? e0.x : e0.y, b_g0 = red0 ? e0.y : e0.x;
    const float r_g1 = red0 ? e1.y : e1.x, b_g1 = red0 ? e1.x : e1.y;
    if (A == 0) {
        finish_x2(make_float2(r_a, r_g0), make_float2(gc_a, gc_0), make_float2(b_a, b_g0), d, out[0]);
        finish_x2(make_float2(r_g1, r_b), make_float2(gc_1, gc_b), make_float2(b_g1, b_b), d, out[1]);
    } else {
        finish_x2(make_float2(r_g0, r_a), make_float2(gc_0, gc_a), make_float2(b_g0, b_a), d, out[0]);
        finish_x2(make_float2(r_b, r_g1), make_float2(gc_b, gc_1), make_float2(b_b, b_g1), d, out[1]);
    }
}

}  // namespace

// PRE: the green pass reads the per-sensel noise terms staged in shared
// memory instead of evaluating them for each neighbour. Valid when width and
// height are both at least 4: every neighbour the green pass reads past a
// picture edge is then replaced by mirror() (src/demosaic.rs:547-557), so
// each neighbour slot holds a sensel of the site type the slot's clip limit
// assumes (green at distance 1, the centre's colour at distance 2). Frames 2
// sensels wide or tall keep the direct evaluation.
// Four CTAs per SM (64 registers a thread): the kernel is bound by
// instruction issue and loses more to three CTAs' fewer warps than it gains
// from the registers it would spill less.
template <bool PRE, class T, bool FAST>
__global__ void __launch_bounds__(T::kThreads, T::kMinBlocks) k_develop(const __grid_constant__ CUtensorMap codes_map,
                                                                     DevelopDesc d) {
    constexpr int TW = T::TW, TH = T::TH, NW = T::NW, NH = T::NH, GW = T::GW, GH = T::GH;
    constexpr int kDevThreads = T::kThreads, kBoxW = T::kBoxW, kBoxX = T::kBoxX;
    __shared__ __align__(16) DevShared<T> S;
    __shared__ __align__(128) uint16_t box[NH][kBoxW];
    __shared__ __align__(8) uint64_t box_bar;
    // Only the tiles a mask selects (the learned develop's fallback tiles).
    if (d.tile_mask && !d.tile_mask[blockIdx.y * gridDim.x + blockIdx.x]) return;
    const int tid = threadIdx.x;
    const int w = d.w, h = d.h;
    const int x0 = blockIdx.x * TW, y0 = blockIdx.y * TH;
    // Tiles whose halo lies inside the picture (no clamping) load their code
    // values with one TMA box; the others clamp each coordinate.
    const bool tma = d.use_tma && x0 >= 3 && x0 + TW + 3 <= w && y0 >= 3 && y0 + TH + 3 <= h;
    const uint32_t bar = smem_addr(&box_bar);
    if (tid < 8) {
        S.c0[tid] = d.curve_c0[tid];
        S.cd[tid] = d.curve_delta[tid];
    }
    if (tma && tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%1], %0;" ::"r"(uint32_t(sizeof(box))), "r"(bar)
                     : "memory");
        // The code values are read once here: an evict-first L2 policy on
        // the load leaves L2 to the next frame's decode beside.
        uint64_t policy;
        asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(policy));
        asm volatile(
            "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1, "
            "{%3, %4}], [%2], %5;" ::"r"(smem_addr(&box[0][0])),
            "l"(reinterpret_cast<uint64_t>(&codes_map)), "r"(bar), "r"(x0 - 8), "r"(y0 - 3), "l"(policy)
            : "memory");
    }
    __syncthreads();
    // A box that has not landed within a second (it always should) leaves the
    // tile to the clamped loads, which give the same values.
    const bool staged = tma && bar_wait(bar, 1000000000ull);
    const Noise nz{d.noise[0], d.noise[1], d.noise[2]};
    const int red_row = d.cfa >> 1, red_col = d.cfa & 1;
    // 1. Normalized values, coordinates clamped to the picture as the green
    //    pass clamps them (src/demosaic.rs:370-375, 499).
    // Two horizontally adjacent values a thread, as the lanes of pairs.
    for (int i = tid; i < NH * (NW / 2); i += kDevThreads) {
        const int ty = i / (NW / 2), tx = 2 * (i - ty * (NW / 2));
        const int y = min(max(y0 - 3 + ty, 0), h - 1);
        const int xa = min(max(x0 - 3 + tx, 0), w - 1), xb = min(max(x0 - 2 + tx, 0), w - 1);
        uint32_t ca, cb;
        if (staged) {
            ca = box[ty][tx + kBoxX];
            cb = box[ty][tx + 1 + kBoxX];
        } else {
            const uint16_t* row = d.codes + size_t(y) * d.stride;
            ca = __ldg(row + xa);
            cb = __ldg(row + xb);
        }
        const int32_t la = int32_t(curve_apply(S.c0, S.cd, ca)), lb = int32_t(curve_apply(S.c0, S.cd, cb));
        const float2 v = mul2(bc(d.one_over_range), make_float2(__int2float_rn(la - d.black), __int2float_rn(lb - d.black)));
        *reinterpret_cast<float2*>(&S.nrm[ty][tx]) = v;
        if (PRE) {
            const bool red_line = (y & 1) == red_row;
            const int rbc = red_line ? red_col : 1 - red_col;
            const float rlim = red_line ? d.clip[0] : d.clip[1];
            const float lima = (xa & 1) == rbc ? rlim : 1.0f, limb = (xb & 1) == rbc ? rlim : 1.0f;
            const float2 var = variance2(make_float2(fminf(v.x, lima), fminf(v.y, limb)), d.green_off, nz);
            *reinterpret_cast<float2*>(&S.gvar[ty][tx]) = var;
            *reinterpret_cast<float2*>(&S.gsd[ty][tx]) = FAST ? sqrt_rn_x2(var) : make_float2(rt(var.x), rt(var.y));
        }
    }
    __syncthreads();
    if (tma && !staged && tid == 0) bar_wait(bar, 1000000000ull);  // a late box lands before the CTA ends
    // mirror() changes a neighbour only for sites within 2 sensels of a
    // picture edge; the green-pass sites of a tile lie within [x0 - 1,
    // x0 + TW] x [y0 - 1, y0 + TH], so tiles clear of the edges skip it
    // (a branch uniform over the block).
    const bool near_edge = x0 < 3 || x0 + TW + 3 > w || y0 < 3 || y0 + TH + 3 > h;
    // 2. Green pass on the region (the tile plus a 1-sensel halo).
    // One site (gy, gx) of the region (src/demosaic.rs:481-541); the region
    // row gy is picture row y0 - 1 + gy, the column gx picture column
    // x0 - 1 + gx.
    auto one_site = [&](int gy, int gx, bool rbsite) {
        const int y = y0 - 1 + gy;
        const bool phase = (y & 1) == red_row;
        const int x = x0 - 1 + gx;
        if (y < 0 || y >= h || x < 0 || x >= w) return;
        const int ty = gy + 2, tx = gx + 2;  // nrm coordinates
        const float centre = S.nrm[ty][tx];
        float rbv = 0.0f, gv_out = centre;
        if (rbsite) {
            const float clip = phase ? d.clip[0] : d.clip[1];
            const float c = fminf(centre, clip);
            const float bs = d.green_off;
            float hh[4] = {fminf(S.nrm[ty][tx - 1], 1.0f), fminf(S.nrm[ty][tx + 1], 1.0f),
                           fminf(S.nrm[ty][tx - 2], clip), fminf(S.nrm[ty][tx + 2], clip)};
            float vv[4] = {fminf(S.nrm[ty - 1][tx], 1.0f), fminf(S.nrm[ty + 1][tx], 1.0f),
                           fminf(S.nrm[ty - 2][tx], clip), fminf(S.nrm[ty + 2][tx], clip)};
            if (near_edge) {
                mirror(hh, x, w, c);
                mirror(vv, y, h, c);
            }
            float var_h[4], var_v[4], sd_h[4], sd_v[4];
            float sdc;
            if (PRE) {
                // The same neighbours' precomputed terms, permuted by the
                // same mirror() with the centre's terms standing for c.
                const float vc = S.gvar[ty][tx];
                sdc = S.gsd[ty][tx];
                var_h[0] = S.gvar[ty][tx - 1]; var_h[1] = S.gvar[ty][tx + 1];
                var_h[2] = S.gvar[ty][tx - 2]; var_h[3] = S.gvar[ty][tx + 2];
                var_v[0] = S.gvar[ty - 1][tx]; var_v[1] = S.gvar[ty + 1][tx];
                var_v[2] = S.gvar[ty - 2][tx]; var_v[3] = S.gvar[ty + 2][tx];
                sd_h[0] = S.gsd[ty][tx - 1]; sd_h[1] = S.gsd[ty][tx + 1];
                sd_h[2] = S.gsd[ty][tx - 2]; sd_h[3] = S.gsd[ty][tx + 2];
                sd_v[0] = S.gsd[ty - 1][tx]; sd_v[1] = S.gsd[ty + 1][tx];
                sd_v[2] = S.gsd[ty - 2][tx]; sd_v[3] = S.gsd[ty + 2][tx];
                if (near_edge) {
                    mirror(var_h, x, w, vc);
                    mirror(var_v, y, h, vc);
                    mirror(sd_h, x, w, sdc);
                    mirror(sd_v, y, h, sdc);
                }
            } else {
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    var_h[i] = variance(hh[i], bs, nz);
                    var_v[i] = variance(vv[i], bs, nz);
                    sd_h[i] = rt(var_h[i]);
                    sd_v[i] = rt(var_v[i]);
                }
                sdc = rt(variance(c, bs, nz));
            }
            const float sums0 = add(hh[0], hh[1]), sums1 = add(vv[0], vv[1]);
            const float sums2 = add(hh[2], hh[3]), sums3 = add(vv[2], vv[3]);
            float ratio0 = 0.0f, ratio1 = 0.0f;
            if (c > sdc) {
                const float t0 = add(mul(c, 2.0f), sums2), t1 = add(mul(c, 2.0f), sums3);
                const float t2 = add(mul(c, -2.0f), sums2), t3 = add(mul(c, -2.0f), sums3);
#pragma unroll
                for (int dir = 0; dir < 2; dir++) {
                    const float* dd = dir == 0 ? hh : vv;
                    const float* sd = dir == 0 ? sd_h : sd_v;
                    const float a = sub(dd[0], dd[1]);
                    const float b = sub(dd[2], dd[3]);
                    const bool any = mul(a, b) > 0.0f || mul(sub(dd[2], c), sub(dd[3], c)) > 0.0f ||
                                     add(sd[0], sd[1]) > fabsf(a) || add(sd[2], sd[3]) > fabsf(b);
                    const bool all = dd[0] > sd[0] && dd[1] > sd[1] && dd[2] > sd[2] && dd[3] > sd[3];
                    if (any && all) {
                        if (dir == 0)
                            ratio0 = dv(t2, mul(t0, 2.0f));
                        else
                            ratio1 = dv(t3, mul(t1, 2.0f));
                    }
                }
            }
            const float gh = mul(mul(sums0, 0.5f), sub(1.0f, ratio0));
            const float gvv = mul(mul(sums1, 0.5f), sub(1.0f, ratio1));
            const float dh0 = sub(hh[0], gh), dh1 = sub(hh[1], gh), dh2 = sub(hh[2], c), dh3 = sub(hh[3], c);
            const float dv0 = sub(vv[0], gvv), dv1 = sub(vv[1], gvv), dv2 = sub(vv[2], c), dv3 = sub(vv[3], c);
            const float eh = add(dot4(dh0, dh1, dh2, dh3, dh0, dh1, dh2, dh3), add(var_h[0], var_h[1]));
            const float ev = add(dot4(dv0, dv1, dv2, dv3, dv0, dv1, dv2, dv3), add(var_v[0], var_v[1]));
            rbv = c;
            gv_out = add(gvv, dv(mul(sub(gh, gvv), ev), add(eh, ev)));
            const float vxx = variance(rbv, d.chroma_off, nz);
            S.vx[gy][gx] = vxx;
            S.sx[gy][gx] = rt(vxx);
        }
        S.rb[gy][gx] = rbv;
        S.gr[gy][gx] = gv_out;
        S.sg[gy][gx] = rt(variance(gv_out, d.chroma_off, nz));
    };
    // First green column mod 2 of region row gy (x0 and y0 are even).
    auto first_of = [&](int gy) {
        const bool phase = ((gy + 1) & 1) == red_row;
        return phase ? red_col : 1 - red_col;
    };
    if (PRE && !near_edge) {
        // Tiles clear of the edges: no mirror(), every site inside the
        // picture. Two sites at a time as the lanes of pairs, lane x in
        // region row gy0, lane y in row gy0 + 1 (the other colour).
        auto site_pair = [&](bool rbsite, int gy0, int gx0, int gx1) {
            const int gy1 = gy0 + 1;
            const int ty0 = gy0 + 2, tx0 = gx0 + 2, ty1 = gy1 + 2, tx1 = gx1 + 2;  // nrm coordinates
            const bool phase0 = ((gy0 + 1) & 1) == red_row;
            const float2 clip = phase0 ? make_float2(d.clip[0], d.clip[1]) : make_float2(d.clip[1], d.clip[0]);
            const float2 centre = make_float2(S.nrm[ty0][tx0], S.nrm[ty1][tx1]);
            float2 rbv = make_float2(0.0f, 0.0f), gv_out = centre;
            if (rbsite) {
                const float2 c = make_float2(fminf(centre.x, clip.x), fminf(centre.y, clip.y));
                const float2 sdc = make_float2(S.gsd[ty0][tx0], S.gsd[ty1][tx1]);
                const bool condx = c.x > sdc.x, condy = c.y > sdc.y;
                float2 g[2], e[2];
    #pragma unroll
                for (int dir = 0; dir < 2; dir++) {
                    // Neighbours at distance 1 (green) and 2 (the centre's
                    // colour), in the order of src/demosaic.rs:499-505.
                    const int oy[4] = {dir ? -1 : 0, dir ? 1 : 0, dir ? -2 : 0, dir ? 2 : 0};
                    const int ox[4] = {dir ? 0 : -1, dir ? 0 : 1, dir ? 0 : -2, dir ? 0 : 2};
                    float2 dd[4], sd[4];
    #pragma unroll
                    for (int n = 0; n < 4; n++) {
                        const float lx = n < 2 ? 1.0f : clip.x, ly = n < 2 ? 1.0f : clip.y;
                        dd[n] = make_float2(fminf(S.nrm[ty0 + oy[n]][tx0 + ox[n]], lx),
                                            fminf(S.nrm[ty1 + oy[n]][tx1 + ox[n]], ly));
                        sd[n] = make_float2(S.gsd[ty0 + oy[n]][tx0 + ox[n]], S.gsd[ty1 + oy[n]][tx1 + ox[n]]);
                    }
                    const float2 sums01 = add2(dd[0], dd[1]), sums23 = add2(dd[2], dd[3]);
                    float2 ratio = make_float2(0.0f, 0.0f);
                    if (condx | condy) {
                        const float2 t0 = add2(mul2(c, bc(2.0f)), sums23);
                        const float2 t2 = add2(mul2(c, bc(-2.0f)), sums23);
                        const float2 a = sub2(dd[0], dd[1]), b = sub2(dd[2], dd[3]);
                        const float2 ab = mul2(a, b), pc = mul2(sub2(dd[2], c), sub2(dd[3], c));
                        const float2 s01 = add2(sd[0], sd[1]), s23 = add2(sd[2], sd[3]);
                        const bool anyx = (ab.x > 0.0f) | (pc.x > 0.0f) | (s01.x > fabsf(a.x)) | (s23.x > fabsf(b.x));
                        const bool anyy = (ab.y > 0.0f) | (pc.y > 0.0f) | (s01.y > fabsf(a.y)) | (s23.y > fabsf(b.y));
                        const bool allx = (dd[0].x > sd[0].x) & (dd[1].x > sd[1].x) & (dd[2].x > sd[2].x) &
                                          (dd[3].x > sd[3].x);
                        const bool ally = (dd[0].y > sd[0].y) & (dd[1].y > sd[1].y) & (dd[2].y > sd[2].y) &
                                          (dd[3].y > sd[3].y);
                        const float2 den = mul2(t0, bc(2.0f));
                        const bool px = condx & anyx & allx, py = condy & anyy & ally;
                        if (FAST) {
                            if (px | py) {
                                const float2 q = div_rn_x2(t2, den);
                                ratio = make_float2(px ? q.x : 0.0f, py ? q.y : 0.0f);
                            }
                        } else {
                            if (px) ratio.x = dv(t2.x, den.x);
                            if (py) ratio.y = dv(t2.y, den.y);
                        }
                    }
                    g[dir] = mul2(mul2(sums01, bc(0.5f)), sub2(bc(1.0f), ratio));
                    const float2 e0 = sub2(dd[0], g[dir]), e1 = sub2(dd[1], g[dir]), e2 = sub2(dd[2], c),
                                 e3 = sub2(dd[3], c);
                    const float2 va = add2(make_float2(S.gvar[ty0 + oy[0]][tx0 + ox[0]], S.gvar[ty1 + oy[0]][tx1 + ox[0]]),
                                           make_float2(S.gvar[ty0 + oy[1]][tx0 + ox[1]], S.gvar[ty1 + oy[1]][tx1 + ox[1]]));
                    e[dir] = add2(dot4x2(e0, e1, e2, e3, e0, e1, e2, e3), va);
                }
                rbv = c;
                const float2 num = mul2(sub2(g[0], g[1]), e[1]), den = add2(e[0], e[1]);
                // This quotient stays div.rn in both variants: with the paired
                // division here the develop was measured not bit-exact
                // (about one output in 20,000 off by an ulp or a few),
                // although the division equals div.rn on every operand pair
                // its tests check; the cause was not found.
                gv_out = add2(g[1], make_float2(dv(num.x, den.x), dv(num.y, den.y)));
                const float2 vxx = variance2(rbv, d.chroma_off, nz);
                S.vx[gy0][gx0] = vxx.x;
                S.vx[gy1][gx1] = vxx.y;
                const float2 sxx = FAST ? sqrt_rn_x2(vxx) : make_float2(rt(vxx.x), rt(vxx.y));
                S.sx[gy0][gx0] = sxx.x;
                S.sx[gy1][gx1] = sxx.y;
            }
            const float2 vg = variance2(gv_out, d.chroma_off, nz);
            S.rb[gy0][gx0] = rbv.x;
            S.rb[gy1][gx1] = rbv.y;
            S.gr[gy0][gx0] = gv_out.x;
            S.gr[gy1][gx1] = gv_out.y;
            const float2 sgg = FAST ? sqrt_rn_x2(vg) : make_float2(rt(vg.x), rt(vg.y));
            S.sg[gy0][gx0] = sgg.x;
            S.sg[gy1][gx1] = sgg.y;
        };
        // Each thread's quad of the tile (region rows 2 qy + 1, 2 qy + 2,
        // columns 2 qx + 1, 2 qx + 2): its red/blue pair, the heavy work,
        // one per thread.
        {
            const int gy0 = 2 * (tid / T::QW) + 1, gxq = 2 * (tid % T::QW) + 1;
            const int f0 = first_of(gy0);
            site_pair(true, gy0, gxq + f0, gxq + 1 - f0);
        }
        // Then the 66 red/blue sites of the halo, one a thread, and the
        // green sites as pairs (rows 2i and 2i + 1 of region quad (i, j)).
        constexpr int kHalo = 2 * (GW / 2) + 2 * (TH / 2), kGreenPairs = (GH / 2) * (GW / 2);
        const int g1 = first_of(1);
        // The halo's red/blue sites to the first kHalo threads, the (light)
        // green pairs to the others, so that no thread takes a halo site and
        // a green pair.
        static_assert(kHalo < kDevThreads, "a halo site a thread");
        if (tid < kHalo) {
            const int u = tid;
            int gy, gx;
            if (u < GW / 2) {  // region row 0
                gy = 0;
                gx = 2 * u + 1 - first_of(0);
            } else if (u < GW) {  // region row GH - 1
                gy = GH - 1;
                gx = 2 * (u - GW / 2) + 1 - first_of(GH - 1);
            } else if (u < GW + TH / 2) {  // column 0: rows whose first green column is odd
                gy = 1 + 2 * (u - GW) + (g1 == 1 ? 0 : 1);
                gx = 0;
            } else {  // column GW - 1: rows whose first green column is even
                gy = 1 + 2 * (u - GW - TH / 2) + (g1 == 0 ? 0 : 1);
                gx = GW - 1;
            }
            one_site(gy, gx, true);
        } else {
            for (int uu = tid - kHalo; uu < kGreenPairs; uu += kDevThreads - kHalo) {
                const int i = uu / (GW / 2), j = uu - i * (GW / 2);
                const int f0 = first_of(2 * i);
                site_pair(false, 2 * i, 2 * j + f0, 2 * j + 1 - f0);
            }
        }
    } else {
        // Tiles at the picture edges: one site a thread, red/blue sites
        // first (the heavy ones), 17 per region row, then green sites.
        for (int k = tid; k < GH * (GW / 2) * 2; k += kDevThreads) {
            const bool rbsite = k < GH * (GW / 2);
            const int kk = rbsite ? k : k - GH * (GW / 2);
            const int gy = kk / (GW / 2), j = kk - gy * (GW / 2);
            const int first = first_of(gy);
            one_site(gy, 2 * j + (rbsite ? 1 - first : first), rbsite);
        }
    }
    __syncthreads();
    // 3. Chroma (+ matrix) per quad.
    const int qx = tid % T::QW, qy = tid / T::QW;
    const int xb = x0 + 2 * qx, yb = y0 + 2 * qy;
    if (xb >= w || yb >= h) return;
    if (!near_edge) {
        // Quad rows start on even picture rows (y0 and 2 * qy are even).
        const bool red0 = red_row == 0;
        float2 o2[2][3];
        if ((red0 ? red_col : 1 - red_col) == 0)
            chroma_quad<T, 0, FAST>(S, 2 * qy + 1, 2 * qx + 1, red0, d, o2);
        else
            chroma_quad<T, 1, FAST>(S, 2 * qy + 1, 2 * qx + 1, red0, d, o2);
        // The planes are written once and not read here again: streaming
        // stores (evict first) leave L2 to the next frame's decode beside.
#pragma unroll
        for (int dy = 0; dy < 2; dy++) {
            const size_t p = size_t(yb + dy) * w + xb;
            if (d.layout == PRR_PLANAR) {
                __stcs(reinterpret_cast<float2*>(d.r + p), o2[dy][0]);
                __stcs(reinterpret_cast<float2*>(d.g + p), o2[dy][1]);
                __stcs(reinterpret_cast<float2*>(d.b + p), o2[dy][2]);
            } else {
                float2* o = reinterpret_cast<float2*>(d.r + 3 * p);
                __stcs(o, make_float2(o2[dy][0].x, o2[dy][1].x));
                __stcs(o + 1, make_float2(o2[dy][2].x, o2[dy][0].y));
                __stcs(o + 2, make_float2(o2[dy][1].y, o2[dy][2].y));
            }
        }
        return;
    }
    float out[2][2][3];
#pragma unroll
    for (int dy = 0; dy < 2; dy++) {
        const int y = yb + dy;
        const int ym = y > 0 ? y - 1 : y + 1, yp = y < h - 1 ? y + 1 : y - 1;
        const int gy = y - y0 + 1, gym = ym - y0 + 1, gyp = yp - y0 + 1;
        const bool on_red_row = (y & 1) == red_row;
        const int rb_col = on_red_row ? red_col : 1 - red_col;
#pragma unroll
        for (int dx = 0; dx < 2; dx++) {
            const int x = xb + dx;
            const int xm = x > 0 ? x - 1 : x + 1, xp = x < w - 1 ? x + 1 : x - 1;
            const int gx = x - x0 + 1, gxm = xm - x0 + 1, gxp = xp - x0 + 1;
            const float c = S.rb[gy][gx], g = S.gr[gy][gx], cs = S.sg[gy][gx];
            float r, b;
            if ((x & 1) == rb_col) {
                const int ny[4] = {gym, gyp, gym, gyp}, nx[4] = {gxm, gxm, gxp, gxp};
                float xx[4], gg[4], vx[4], sx[4], sg[4];
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    xx[i] = S.rb[ny[i]][nx[i]];
                    gg[i] = S.gr[ny[i]][nx[i]];
                    vx[i] = S.vx[ny[i]][nx[i]];
                    sx[i] = S.sx[ny[i]][nx[i]];
                    sg[i] = S.sg[ny[i]][nx[i]];
                }
                const float e = estimate(xx, gg, vx, sx, sg, g, cs);
                r = on_red_row ? c : e;
                b = on_red_row ? e : c;
            } else {
                // Each of two opposite neighbours counts twice.
                auto pair = [&](int uy, int ux, int vy, int vx_) {
                    const float xu = S.rb[uy][ux], xv = S.rb[vy][vx_];
                    const float gu = S.gr[uy][ux], gv = S.gr[vy][vx_];
                    const float vu = S.vx[uy][ux], vvv = S.vx[vy][vx_];
                    const float su = S.sx[uy][ux], sv = S.sx[vy][vx_];
                    const float tu = S.sg[uy][ux], tv = S.sg[vy][vx_];
                    return estimate2(xu, xv, gu, gv, vu, vvv, su, sv, tu, tv, g, cs);
                };
                const float eh = pair(gy, gxm, gy, gxp);
                const float ev = pair(gym, gx, gyp, gx);
                r = on_red_row ? eh : ev;
                b = on_red_row ? ev : eh;
            }
            float rr = fminf(mul(r, d.wb[0]), 1.0f);
            float gg = fminf(g, 1.0f);
            float bb = fminf(mul(b, d.wb[1]), 1.0f);
            if (d.has_matrix) {
                const float m0 = fma_(bb, d.m[2], fma_(rr, d.m[0], mul(gg, d.m[1])));
                const float m1 = fma_(bb, d.m[5], fma_(rr, d.m[3], mul(gg, d.m[4])));
                const float m2 = fma_(bb, d.m[8], fma_(rr, d.m[6], mul(gg, d.m[7])));
                rr = m0;
                gg = m1;
                bb = m2;
            }
            out[dy][dx][0] = rr;
            out[dy][dx][1] = gg;
            out[dy][dx][2] = bb;
        }
    }
#pragma unroll
    for (int dy = 0; dy < 2; dy++) {
        const size_t p = size_t(yb + dy) * w + xb;
        if (d.layout == PRR_PLANAR) {
            __stcs(reinterpret_cast<float2*>(d.r + p), make_float2(out[dy][0][0], out[dy][1][0]));
            __stcs(reinterpret_cast<float2*>(d.g + p), make_float2(out[dy][0][1], out[dy][1][1]));
            __stcs(reinterpret_cast<float2*>(d.b + p), make_float2(out[dy][0][2], out[dy][1][2]));
        } else {
            float2* o = reinterpret_cast<float2*>(d.r + 3 * p);
            __stcs(o, make_float2(out[dy][0][0], out[dy][0][1]));
            __stcs(o + 1, make_float2(out[dy][0][2], out[dy][1][0]));
            __stcs(o + 2, make_float2(out[dy][1][1], out[dy][1][2]));
        }
    }
}

// Frame::linearize_into (src/decoder.rs:197-216), curve of src/curve.rs:14-24.
// A CTA of 256 threads takes 1024 consecutive chunks of eight sensels
// (16 bytes): each thread issues its four 16-byte loads before it
// converts and stores any of them, so that enough bytes are in flight to
// keep HBM busy (one chunk a thread measured 0.37 of the HBM peak). FLAT:
// rows are packed (stride == width, a multiple of 8, 16-byte aligned
// output), so chunk k is bytes [16 k, 16 k + 16) of input and output alike.
struct CurveDesc {
    uint32_t c0[8], cd[8];
};
constexpr int kLinChunks = 4;  // chunks of 8 sensels a thread

template <bool FLAT>
__global__ void __launch_bounds__(256) k_linearize(const uint16_t* __restrict__ codes, uint32_t stride, int w, int h,
                                                   CurveDesc curve, uint16_t* __restrict__ out, int vec_out,
                                                   size_t nchunks) {
    __shared__ uint32_t c0[8], cd[8];
    if (threadIdx.x < 8) {
        c0[threadIdx.x] = curve.c0[threadIdx.x];
        cd[threadIdx.x] = curve.cd[threadIdx.x];
    }
    __syncthreads();
    const size_t first = size_t(blockIdx.x) * (blockDim.x * kLinChunks) + threadIdx.x;
    const int cpr = (w + 7) / 8;
    uint4 raw[kLinChunks];
    int xcs[kLinChunks], ys[kLinChunks];
#pragma unroll
    for (int k = 0; k < kLinChunks; k++) {
        const size_t idx = first + size_t(k) * blockDim.x;
        raw[k] = make_uint4(0, 0, 0, 0);
        ys[k] = h;
        xcs[k] = 0;
        if (idx >= nchunks) continue;
        if (FLAT) {
            raw[k] = __ldcs(reinterpret_cast<const uint4*>(codes) + idx);
            ys[k] = 0;
        } else {
            const int y = int(idx / cpr), xc = int(idx - size_t(y) * cpr) * 8;
            ys[k] = y;
            xcs[k] = xc;
            if (xc + 8 <= w) raw[k] = __ldcs(reinterpret_cast<const uint4*>(codes + size_t(y) * stride + xc));
        }
    }
#pragma unroll
    for (int k = 0; k < kLinChunks; k++) {
        const size_t idx = first + size_t(k) * blockDim.x;
        if (idx >= nchunks) continue;
        if (FLAT) {
            const uint16_t* in = reinterpret_cast<const uint16_t*>(&raw[k]);
            __align__(16) uint16_t v[8];
#pragma unroll
            for (int e = 0; e < 8; e++) v[e] = uint16_t(curve_apply(c0, cd, in[e]));
            reinterpret_cast<uint4*>(out)[idx] = *reinterpret_cast<const uint4*>(v);
            continue;
        }
        const int y = ys[k], xc = xcs[k];
        const uint16_t* src = codes + size_t(y) * stride + xc;
        uint16_t* dst = out + size_t(y) * w + xc;
        if (xc + 8 <= w) {
            const uint16_t* in = reinterpret_cast<const uint16_t*>(&raw[k]);
            __align__(16) uint16_t v[8];
#pragma unroll
            for (int e = 0; e < 8; e++) v[e] = uint16_t(curve_apply(c0, cd, in[e]));
            if (vec_out) {
                *reinterpret_cast<uint4*>(dst) = *reinterpret_cast<const uint4*>(v);
            } else {
#pragma unroll
                for (int e = 0; e < 8; e++) dst[e] = v[e];
            }
        } else {
            for (int e = 0; xc + e < w; e++) dst[e] = uint16_t(curve_apply(c0, cd, src[e]));
        }
    }
}

cudaError_t launch_linearize(const uint16_t* codes, uint32_t stride, int w, int h, const uint32_t* c0,
                             const uint32_t* delta, uint16_t* out, cudaStream_t s) {
    const size_t chunks = size_t((w + 7) / 8) * h;
    if (chunks == 0) return cudaSuccess;
    const bool out_aligned = (reinterpret_cast<uintptr_t>(out) & 15) == 0;
    const int vec_out = (w % 8 == 0) && out_aligned;
    const bool flat = vec_out && stride == uint32_t(w) && (reinterpret_cast<uintptr_t>(codes) & 15) == 0;
    const size_t per_block = size_t(256) * kLinChunks;
    const unsigned blocks = unsigned((chunks + per_block - 1) / per_block);
    CurveDesc curve;
    for (int i = 0; i < 8; i++) {
        curve.c0[i] = c0[i];
        curve.cd[i] = delta[i];
    }
    if (flat)
        k_linearize<true><<<blocks, 256, 0, s>>>(codes, stride, w, h, curve, out, vec_out, chunks);
    else
        k_linearize<false><<<blocks, 256, 0, s>>>(codes, stride, w, h, curve, out, vec_out, chunks);
    count_launch();
    return cudaGetLastError();
}

// Diagnostics of the paired division (fastdiv.cuh): quotients of arrays,
// two a thread as the develop computes them; and a count of the pairs
// (a, b), a over all 2^23 significands in [1, 2) and b over the
// significands [b_first, b_first + b_count), whose paired quotient differs
// from div.rn.f32 (one b per CTA), plus the b whose reciprocal does not
// scale exactly over the exponents [-100, 100].
__global__ void k_div_rn_pairs(const float* __restrict__ a, const float* __restrict__ b, float* __restrict__ q,
                               size_t n) {
    const size_t i = 2 * (size_t(blockIdx.x) * blockDim.x + threadIdx.x);
    if (i >= n) return;
    const bool two = i + 1 < n;
    const float2 r = div_rn_x2(make_float2(a[i], two ? a[i + 1] : 1.0f), make_float2(b[i], two ? b[i + 1] : 1.0f));
    q[i] = r.x;
    if (two) q[i + 1] = r.y;
}

__global__ void __launch_bounds__(256) k_div_rn_check(uint32_t b_first, unsigned long long* mismatches) {
    const uint32_t bb = 0x3F800000u | (b_first + blockIdx.x);
    const float bf = __uint_as_float(bb);
    unsigned long long bad = 0;
    // The reciprocal scales exactly with b: 1/(b 2^k) = (1/b) 2^-k for k in
    // [-100, 100], so the pairs of [1, 2) x [1, 2) stand for every exponent.
    if (threadIdx.x <= 200) {
        const int k = int(threadIdx.x) - 100;
        const float bk = __uint_as_float(uint32_t(int32_t(bb) + k * (1 << 23)));
        const float sk = __uint_as_float(uint32_t(127 - k) << 23);  // 2^-k
        const float y = rcp_rn_x2(make_float2(bf, bf)).x, yk = rcp_rn_x2(make_float2(bk, bk)).x;
        bad += __float_as_uint(yk) != __float_as_uint(__fmul_rn(y, sk));
    }
    for (uint32_t m = threadIdx.x; m < (1u << 22); m += blockDim.x) {
        const float a0 = __uint_as_float(0x3F800000u | (2 * m)), a1 = __uint_as_float(0x3F800000u | (2 * m + 1));
        const float2 r = div_rn_x2(make_float2(a0, a1), make_float2(bf, bf));
        bad += (__float_as_uint(r.x) != __float_as_uint(__fdiv_rn(a0, bf))) +
               (__float_as_uint(r.y) != __float_as_uint(__fdiv_rn(a1, bf)));
    }
    if (bad) atomicAdd(mismatches, bad);
}

// Every float with exponent in [e_min, e_max] (one exponent per CTA, the
// significands over its threads, two a thread): count those whose paired
// square root differs from sqrt.rn.f32.
__global__ void __launch_bounds__(256) k_sqrt_rn_check(int e_min, unsigned long long* mismatches) {
    const uint32_t ex = uint32_t(e_min + int(blockIdx.x) + 127) << 23;
    unsigned long long bad = 0;
    for (uint32_t m = blockIdx.y * blockDim.x + threadIdx.x; m < (1u << 22); m += gridDim.y * blockDim.x) {
        const float x0 = __uint_as_float(ex | (2 * m)), x1 = __uint_as_float(ex | (2 * m + 1));
        const float2 r = sqrt_rn_x2(make_float2(x0, x1));
        bad += (__float_as_uint(r.x) != __float_as_uint(__fsqrt_rn(x0))) +
               (__float_as_uint(r.y) != __float_as_uint(__fsqrt_rn(x1)));
    }
    if (bad) atomicAdd(mismatches, bad);
}

cudaError_t launch_sqrt_rn_check(int e_min, int e_max, unsigned long long* mismatches, cudaStream_t s) {
    if (e_min < -126 || e_max > 127 || e_min > e_max) return cudaErrorInvalidValue;
    k_sqrt_rn_check<<<dim3(unsigned(e_max - e_min + 1), 64), 256, 0, s>>>(e_min, mismatches);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_div_rn_pairs(const float* a, const float* b, float* q, size_t n, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    const size_t threads = (n + 1) / 2;
    k_div_rn_pairs<<<unsigned((threads + 255) / 256), 256, 0, s>>>(a, b, q, n);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_div_rn_check(uint32_t b_first, uint32_t b_count, unsigned long long* mismatches,
                                cudaStream_t s) {
    if (b_first >= (1u << 23) || b_count > (1u << 23) - b_first) return cudaErrorInvalidValue;
    // At most 4096 significands of b a launch (2^35 pairs).
    for (uint32_t k = 0; k < b_count; k += 4096) {
        k_div_rn_check<<<std::min(4096u, b_count - k), 256, 0, s>>>(b_first + k, mismatches);
        count_launch();
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

namespace {

// Dynamic shared memory that caps k_develop<PRE, T, FAST> at `ctas` CTAs
// per SM (0: none), found with the occupancy calculator and kept per cap.
template <bool PRE, class T, bool FAST>
cudaError_t develop_reserve(uint32_t ctas, size_t* bytes) {
    *bytes = 0;
    if (ctas == 0) return cudaSuccess;
    // Per device and cap: the pad found, plus one (0: not yet found). The
    // attribute below is set on the device the first time.
    static std::atomic<uint32_t> cache[kMaxDevices][17];
    int dev = 0, per_sm = 0, per_block = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices || ctas > 16) return cudaErrorInvalidValue;
    const uint32_t known = cache[dev][ctas].load(std::memory_order_acquire);
    if (known) {
        *bytes = known - 1;
        return cudaSuccess;
    }
    cudaFuncAttributes fa;
    e = cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&per_block, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k_develop<PRE, T, FAST>);
    if (e != cudaSuccess) return e;
    const size_t fixed = fa.sharedSizeBytes;  // the kernel's static shared memory
    // A block's static plus dynamic shared memory above 48 KB needs the
    // opt-in limit.
    e = cudaFuncSetAttribute(k_develop<PRE, T, FAST>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             int(std::min<size_t>(size_t(per_block) - fixed, size_t(per_sm))));
    if (e != cudaSuccess) return e;
    const size_t step = 1024;
    size_t pad = 0;
    for (;;) {
        int n = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_develop<PRE, T, FAST>, T::kThreads, pad);
        if (e != cudaSuccess) return e;
        if (n <= int(ctas) || pad + fixed + step > size_t(per_block)) break;
        pad += step;
    }
    cache[dev][ctas].store(uint32_t(pad) + 1, std::memory_order_release);
    *bytes = pad;
    return cudaSuccess;
}

template <class T>
cudaError_t launch_develop_shape(DevelopDesc d, cudaStream_t s) {
    dim3 grid((d.w + T::TW - 1) / T::TW, (d.h + T::TH - 1) / T::TH);
    // The code values as a 2-D tensor (rows of the coded width, the
    // picture's height) for the TMA tile loads; a buffer that is not 16-byte
    // aligned, or a map the driver refuses, leaves every tile to the
    // clamped loads.
    alignas(64) CUtensorMap map;
    std::memset(&map, 0, sizeof(map));
    d.use_tma = 0;
    if ((reinterpret_cast<uintptr_t>(d.codes) & 15) == 0 && (d.stride * 2) % 16 == 0 && d.w >= T::TW + 6 &&
        d.h >= T::TH + 6)
        d.use_tma = encode_u16_map_2d(&map, d.codes, d.stride, uint64_t(d.h), uint64_t(d.stride) * 2, T::kBoxW,
                                      T::NH) == cudaSuccess;
    size_t pad = 0;
    cudaError_t e;
    if (d.w >= 4 && d.h >= 4 && develop_fast_division_ok(d)) {
        if ((e = develop_reserve<true, T, true>(d.ctas_per_sm, &pad)) != cudaSuccess) return e;
        k_develop<true, T, true><<<grid, T::kThreads, pad, s>>>(map, d);
    } else if (d.w >= 4 && d.h >= 4) {
        if ((e = develop_reserve<true, T, false>(d.ctas_per_sm, &pad)) != cudaSuccess) return e;
        k_develop<true, T, false><<<grid, T::kThreads, pad, s>>>(map, d);
    } else {
        if ((e = develop_reserve<false, T, false>(d.ctas_per_sm, &pad)) != cudaSuccess) return e;
        k_develop<false, T, false><<<grid, T::kThreads, pad, s>>>(map, d);
    }
    count_launch();
    return cudaGetLastError();
}

}  // namespace

// The paired division (fastdiv.cuh) is exact for operands inside [2^-100,
// 2^100] and quotients inside [2^-120, 2^120], the paired square root on
// [2^-60, 2^60] (every variance lies in [c, 2^43]). Under these parameter bounds
// every quotient of the green and chroma passes of interior tiles is inside
// (the estimates' weight is also checked per site): the noise floor c
// bounds every noise deviation below by sqrt(c) >= 2^-20, so every divisor
// and numerator the passes form once their tests pass is at least
// (2^-20 * 2^-24)^2; normalized values are at most 65535 * one_over_range
// <= 65535, green estimates at most 1.5 times that, variances at most c +
// max(b, a (off + v)^2) <= 2^43. DemosaicParams::new and
// ::with_white_balance always give such parameters (c = 64/3 / range^2 >=
// 2^-28 for range <= 65535; a <= 140; b < 1); other parameters take div.rn
// throughout.
bool develop_fast_division_ok(const DevelopDesc& d) {
    auto in = [](float v, float lo, float hi) { return v >= lo && v <= hi; };  // false for NaN
    return in(d.noise[2], 0x1p-40f, 1.0f) && in(d.noise[0], 0.0f, 256.0f) && in(d.noise[1], 0.0f, 256.0f) &&
           in(d.one_over_range, 0x1p-17f, 1.0f) && in(d.green_off, -65536.0f, 65536.0f) &&
           in(d.chroma_off, -65536.0f, 65536.0f);
}

bool develop_shape_supported(uint32_t tile_w, uint32_t tile_h) {
    return (tile_w == 32 && (tile_h == 32 || tile_h == 16)) || (tile_w == 64 && tile_h == 16);
}

cudaError_t launch_develop(const DevelopDesc& d, cudaStream_t s) {
    if (d.w <= 0 || d.h <= 0) return cudaSuccess;
    const uint32_t tw = d.tile_w ? d.tile_w : 32, th = d.tile_h ? d.tile_h : 32;
    // A tile mask addresses the 32x32 tile grid.
    if (d.tile_mask && (tw != 32 || th != 32)) return cudaErrorInvalidValue;
    if (tw == 32 && th == 32) return launch_develop_shape<Tile32x32>(d, s);
    if (tw == 32 && th == 16) return launch_develop_shape<Tile32x16>(d, s);
    if (tw == 64 && th == 16) return launch_develop_shape<Tile64x16>(d, s);
    return cudaErrorInvalidValue;
}

}  // namespace prr
