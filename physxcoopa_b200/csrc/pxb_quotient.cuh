// pxb_quotient.cuh -- the unit vector d / |d| of a distance constraint: three IEEE single-
// precision quotients by one length, correctly rounded, from one reciprocal.
//
// project_distance (physxcoopa/cloth/cloth_solver.h:119-138) divides each component of d by its
// length; equality with the reference needs each quotient rounded to nearest exactly as an IEEE
// division rounds it. Three full divisions by the same length repeat the same reciprocal work
// three times; this computes the reciprocal once and finishes each quotient with fused
// multiply-adds.
//
// Method (Markstein's: P. Markstein, "Computation of elementary functions on the IBM RISC
// System/6000 processor", IBM J. Res. Develop. 34(1), 1990; "IA-64 and Elementary Functions",
// Prentice Hall 2000, ch. 8). With b the divisor:
//   y  = the hardware reciprocal estimate of b, refined by one Newton-Raphson step,
//        e = 1 - b*y0, y = y0 + e*y0 (each a fused multiply-add, rounded once);
//   q0 = a*y;  r = b*q0 - a (exact under a fused multiply-add);
//   q  = q0 - r*y, rounded once, is a/b rounded to nearest (Markstein's theorem, given y is the
//        correctly rounded reciprocal).
// The remainder is formed as b*q0 - a (not a - b*q0) so that a signed zero numerator keeps its
// sign, as IEEE division keeps it. The pair (dx, dy) goes through the packed two-lane FP32
// instructions of sm_100 (fma.rn.f32x2 / mul.rn.f32x2, each lane rounded as the scalar
// instruction rounds it); dz through the scalar ones.
//
// Range: numerators and divisor are first scaled by 2^64 (exact: a power of two), so a small
// numerator leaves a normal remainder. The method needs a normal quotient: a component whose
// quotient would fall below 2^-100 (0 < |d_i| < 2^-100 |d|) sends the constraint to three IEEE
// divisions, as does a length outside [2^-60, 2^60] (a NaN, a zero length, an edge longer than
// 2^60 m). Zero components stay on the fast path: +-0 / l keeps its sign there. Neither case
// occurs in a cloth of positions away from the origin's subnormal neighbourhood.
//
// Checked on the device against IEEE division (pxb_check_quotients, tests/test_quotient_gpu.py):
// the refined reciprocal is the correctly rounded one for every divisor significand; the
// quotient equals IEEE division for every pair of significands (2^46 pairs, the whole space the
// method's rounding depends on: pxb_check_quotient_significands), and on seeded random
// constraints covering lengths far outside a cloth's, subnormal numerators and signed zeros.
#ifndef PXB_QUOTIENT_CUH
#define PXB_QUOTIENT_CUH

#include <cuda_runtime.h>
#include <stdint.h>

namespace pxb {

// Two-lane FP32 add, multiply and fused multiply-add, each lane rounded to nearest as the scalar
// instruction rounds it (sm_100). The lanes travel as one 64-bit register pair.
__device__ __forceinline__ float2 add2_rn(float2 a, float2 b) {
    float2 d;
    asm("{\n\t.reg .b64 ra, rb, rd;\n\t"
        "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "add.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}
__device__ __forceinline__ float2 mul2_rn(float2 a, float2 b) {
    float2 d;
    asm("{\n\t.reg .b64 ra, rb, rd;\n\t"
        "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "mul.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}
__device__ __forceinline__ float2 fma2_rn(float2 a, float2 b, float2 c) {
    float2 d;
    asm("{\n\t.reg .b64 ra, rb, rc, rd;\n\t"
        "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\tmov.b64 rc, {%6, %7};\n\t"
        "fma.rn.f32x2 rd, ra, rb, rc;\n\tmov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
    return d;
}

// The refined reciprocal of a divisor already scaled into [2^4, 2^124].
__device__ __forceinline__ float rcp_refined(float b) {
    float y0;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y0) : "f"(b));
    const float e = __fmaf_rn(-b, y0, 1.0f);
    return __fmaf_rn(e, y0, y0);
}

// a / b for a scaled numerator na = -a * 2^64 and divisor B = b * 2^64 with y = rcp_refined(B)
// (ny = -y).
__device__ __forceinline__ float quotient_scaled(float na, float B, float ny) {
    const float q0 = na * ny;                 // a*y
    const float r = __fmaf_rn(B, q0, na);     // B*q0 - a, exact
    return __fmaf_rn(r, ny, q0);              // q0 - r*y, rounded once
}
__device__ __forceinline__ float2 quotient_scaled2(float2 na, float2 B, float2 ny) {
    const float2 q0 = mul2_rn(na, ny);
    const float2 r = fma2_rn(B, q0, na);
    return fma2_rn(r, ny, q0);
}

// (nx, ny, nz) = (dx / l, dy / l, dz / l), each rounded to nearest as IEEE division rounds it.
__device__ __forceinline__ void unit3(float dx, float dy, float dz, float l, float& nx, float& ny, float& nz) {
    const float t = l * 0x1p-100f;
    const bool tiny = (fabsf(dx) < t && dx != 0.0f) || (fabsf(dy) < t && dy != 0.0f) || (fabsf(dz) < t && dz != 0.0f);
    if (!(l >= 0x1p-60f && l <= 0x1p60f) || tiny) {
        nx = dx / l;
        ny = dy / l;
        nz = dz / l;
        return;
    }
    const float B = l * 0x1p64f;
    const float y = rcp_refined(B);
    const float yn = -y;
    const float2 q = quotient_scaled2(mul2_rn(make_float2(dx, dy), make_float2(-0x1p64f, -0x1p64f)),
                                      make_float2(B, B), make_float2(yn, yn));
    nx = q.x;
    ny = q.y;
    nz = quotient_scaled(dz * -0x1p64f, B, yn);
}

}  // namespace pxb

#endif  // PXB_QUOTIENT_CUH
