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

__device__ __forceinline__ float rcp_approx(float b) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(b));
    return r;
}

// RN(1/b) for both lanes (b inside the range above; nb = -b).
__device__ __forceinline__ float2 rcp_rn_x2(float2 b, float2 nb) {
    const float2 y0 = make_float2(rcp_approx(b.x), rcp_approx(b.y));
    const float2 e = __ffma2_rn(nb, y0, make_float2(1.0f, 1.0f));
    return __ffma2_rn(y0, e, y0);
}

// RN(a/b) for both lanes (operands inside the range above).
__device__ __forceinline__ float2 div_rn_x2(float2 a, float2 b) {
    const float2 nb = __fmul2_rn(b, make_float2(-1.0f, -1.0f));
    const float2 y = rcp_rn_x2(b, nb);
    const float2 q0 = __fmul2_rn(a, y);
    const float2 r0 = __ffma2_rn(nb, q0, a);
    const float2 q1 = __ffma2_rn(r0, y, q0);
    const float2 r1 = __ffma2_rn(nb, q1, a);
    return __ffma2_rn(r1, y, q1);
}

}  // namespace prr
