// fastdiv.cuh -- correctly rounded f32 division on packed pairs.
//
// The develop's estimates divide two sites' operands at a time (the lanes of
// f32x2 pairs). IEEE division (div.rn.f32) is a scalar subroutine; this is
// the same correctly rounded quotient from the hardware reciprocal
// approximation and packed fused multiply-adds, by the method of Markstein
// (P. Markstein, "Computation of elementary functions on the IBM RISC
// System/6000 processor", IBM J. Res. Dev. 34(1), 1990; also Muller et al.,
// Handbook of Floating-Point Arithmetic, "Newton-Raphson-based division
// with an FMA"):
//   y0 = approximate 1/b                     (rcp.approx, one MUFU op a lane)
//   y  = y0 + y0 (1 - b y0)                  one Newton step: y = RN(1/b)
//   q0 = RN(a y)
//   q1 = q0 + y RN(a - b q0)                 brings q0 within one ulp
//   q  = q1 + y (a - b q1)                   Markstein's correction: RN(a/b)
// Each line is one packed fused multiply-add (or multiply) per two lanes.
// The method is exact only where no operand, quotient or remainder leaves
// the normal range: |a| and |b| in [2^-100, 2^100], |a/b| in [2^-120,
// 2^120]. The develop uses it only under parameters for which every
// quotient it forms lies there (develop_fast_division_ok), and there its
// results equal div.rn.f32 bit for bit: the library's tests check every
// significand pair of [1, 2) x [1, 2) (2^46 pairs; inside that range every
// step is exact under scaling by powers of two), the reciprocal's exact
// scaling over the exponents, random operands across the range and the
// edge classes.
#pragma once

#include <cuda_runtime.h>

namespace prr {

// The packed operations are written as PTX with an explicit .rn rounding
// modifier. An explicit modifier makes the code generator treat each one
// as an IEEE operation of its own: it may not fuse or reorder it with the
// operations around it, so the quotient is exactly the one the steps above
// define, wherever it is inlined.
namespace fastdiv_detail {
__device__ __forceinline__ unsigned long long pack(float2 v) {
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(v.x), "f"(v.y));
    return r;
}
__device__ __forceinline__ float2 unpack(unsigned long long r) {
    float2 v;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(v.x), "=f"(v.y) : "l"(r));
    return v;
}
__device__ __forceinline__ unsigned long long fma_rn(unsigned long long a, unsigned long long b,
                                                     unsigned long long c) {
    unsigned long long r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
    return r;
}
__device__ __forceinline__ unsigned long long mul_rn(unsigned long long a, unsigned long long b) {
    unsigned long long r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ float rcp_approx(float b) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(b));
    return r;
}
__device__ __forceinline__ float rsqrt_approx(float x) {
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
}  // namespace fastdiv_detail

// RN(1/b) for both lanes, b inside the range above (packed; nb = -b).
__device__ __forceinline__ unsigned long long rcp_rn_x2_packed(float2 b, unsigned long long nb) {
    using namespace fastdiv_detail;
    const unsigned long long y0 = pack(make_float2(rcp_approx(b.x), rcp_approx(b.y)));
    const unsigned long long e = fma_rn(nb, y0, pack(make_float2(1.0f, 1.0f)));
    return fma_rn(y0, e, y0);
}

__device__ __forceinline__ float2 rcp_rn_x2(float2 b) {
    using namespace fastdiv_detail;
    return unpack(rcp_rn_x2_packed(b, pack(make_float2(-b.x, -b.y))));
}

// RN(a/b) for both lanes (operands inside the range above).
__device__ __forceinline__ float2 div_rn_x2(float2 a, float2 b) {
    using namespace fastdiv_detail;
    const unsigned long long pa = pack(a);
    const unsigned long long nb = pack(make_float2(-b.x, -b.y));
    const unsigned long long y = rcp_rn_x2_packed(b, nb);
    const unsigned long long q0 = mul_rn(pa, y);
    const unsigned long long r0 = fma_rn(nb, q0, pa);
    const unsigned long long q1 = fma_rn(r0, y, q0);
    const unsigned long long r1 = fma_rn(nb, q1, pa);
    return unpack(fma_rn(r1, y, q1));
}

// RN(sqrt(x)) for both lanes, x in [2^-60, 2^60], by the same method
// (Markstein): from y0 = approximate 1/sqrt(x), g = RN(x y0) ~ sqrt(x) and
// h = y0 / 2 ~ 1/(2 sqrt(x)); one coupled Newton step r = 0.5 - g h,
// g1 = g + g r, h1 = h + h r; then the residual correction
// s = g1 + h1 (x - g1 g1). Every float of that range is checked against
// sqrt.rn.f32 by the library's tests (prr_sqrt_rn_check).
__device__ __forceinline__ float2 sqrt_rn_x2(float2 x) {
    using namespace fastdiv_detail;
    const unsigned long long px = pack(x);
    const unsigned long long y0 = pack(make_float2(rsqrt_approx(x.x), rsqrt_approx(x.y)));
    const unsigned long long g = mul_rn(px, y0);
    const unsigned long long h = mul_rn(y0, pack(make_float2(0.5f, 0.5f)));
    const unsigned long long ng = mul_rn(g, pack(make_float2(-1.0f, -1.0f)));
    const unsigned long long r = fma_rn(ng, h, pack(make_float2(0.5f, 0.5f)));
    const unsigned long long g1 = fma_rn(g, r, g);
    const unsigned long long h1 = fma_rn(h, r, h);
    const unsigned long long ng1 = mul_rn(g1, pack(make_float2(-1.0f, -1.0f)));
    const unsigned long long d = fma_rn(ng1, g1, px);
    return unpack(fma_rn(d, h1, g1));
}

}  // namespace prr
