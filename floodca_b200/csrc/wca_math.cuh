// Rounding-faithful math for the WCA face and cell formulas on sm_100a.
//
// The reference evaluates hf^(2/3) as (real)cbrt((double)hf*hf), the critical
// velocity as (real)sqrt((double)g*hf) and the Manning slope term as
// (real)sqrt((double)S) (FloodCA src/kernels/physics.h:19-24, 105-110,
// 205-207). For float `real` each of these is one correctly rounded float of
// an exactly representable double argument. The helpers below produce that
// same float without double-precision math on the common path:
//
//  * cbrt_sq_rn: float-pair Newton step on a hardware log2/exp2 estimate,
//    then a test of the rounding residual; inputs whose result lies within
//    2^-12 ulp of a rounding midpoint (about 1 in 2000) take an exact
//    midpoint test in double (sign of m^3 - hf^2 by one fused multiply-add).
//  * min_vcr: min(v, RN(sqrt(g*hf))) decided by an exact comparison of v*v
//    with g*hf as float pairs; the square root itself is only evaluated when
//    the critical cap applies, by a float-pair correction of sqrtf (double
//    only within 2^-12 ulp of a rounding midpoint).
//  * sqrt of a float argument: IEEE sqrtf already equals (float)sqrt((double)x).
//
// Build this code with --fmad=false so plain a*b+c stays two rounded ops.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace fcab {

__device__ __forceinline__ float lg2_approx(float x)
{
    float y;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ float ex2_approx(float x)
{
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ float rcp_approx(float x)
{
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ float rsqrt_approx(float x)
{
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Branch-free correctly rounded float operations for normal-range operands
// (the face formulas keep every operand well inside the normal range; the
// callers guard the rest). Each is a one-step Newton/Markstein correction of
// the hardware approximation, checked bit for bit against the IEEE
// operations over whole binades by the GPU tests (fcab_math_probe 4-6).

// RN(1/x), x normal.
__device__ __forceinline__ float rcp_nr(float x)
{
    const float y = rcp_approx(x);
    const float e = __fmaf_rn(-x, y, 1.0f);
    return __fmaf_rn(e, y, y);
}

// RN(a/b) given rb = RN(1/b) (Markstein: q within 1 ulp of a/b, rb within
// half an ulp of 1/b, r = a - b*q exact, then q + r*rb rounds to a/b).
__device__ __forceinline__ float div_mk(float a, float b, float rb)
{
    const float q = __fmul_rn(a, rb);
    const float r = __fmaf_rn(-q, b, a);
    return __fmaf_rn(r, rb, q);
}

// RN(sqrt(x)), x normal and positive.
__device__ __forceinline__ float sqrt_nr(float x)
{
    const float y = rsqrt_approx(x);
    const float s = __fmul_rn(x, y);
    const float h = __fmul_rn(0.5f, y);
    const float r = __fmaf_rn(-s, s, x);
    return __fmaf_rn(r, h, s);
}

// Exact slow path: correct the candidate y towards the side of e by testing
// the rounding midpoint m against the exact value cbrt(c), c = hf^2 (exact in
// double). m has at most 25 significant bits, so m*m is exact in double and
// fma(m*m, m, -c) has the sign of m^3 - c. No exact ties exist (m^3 would need
// about 75 bits, c has at most 48).
static __device__ __noinline__ float cbrt_sq_fix(float hf, float y, float e)
{
    double c = (double)hf * (double)hf;
    if (e > 0.0f) {
        float up = __uint_as_float(__float_as_uint(y) + 1u);
        double m = 0.5 * ((double)y + (double)up);
        if (fma(m * m, m, -c) < 0.0)
            return up;
    } else {
        float dn = __uint_as_float(__float_as_uint(y) - 1u);
        double m = 0.5 * ((double)y + (double)dn);
        if (fma(m * m, m, -c) > 0.0)
            return dn;
    }
    return y;
}

static __device__ __noinline__ float cbrt_sq_wide(float hf)
{
    return (float)cbrt((double)hf * (double)hf);
}

// First phase of cbrt_sq_rn for hf in [2^-20, 2^20]: the candidate y and the
// rounding error e of its correction; returns true when cbrt_sq_fix(hf, y, e)
// must decide (within 2^-12 ulp of a midpoint, or hf out of range).
__device__ __forceinline__ bool cbrt_sq_try(float hf, float &y, float &e)
{
    const float y0 = ex2_approx(__fmul_rn(lg2_approx(hf), 0.666666687f));
    const float c_hi = __fmul_rn(hf, hf);
    const float c_lo = __fmaf_rn(hf, hf, -c_hi);
    const float s_hi = __fmul_rn(y0, y0);
    const float s_lo = __fmaf_rn(y0, y0, -s_hi);
    const float t_hi = __fmul_rn(s_hi, y0);
    float t_lo = __fmaf_rn(s_hi, y0, -t_hi);
    t_lo = __fmaf_rn(s_lo, y0, t_lo);
    const float r = __fadd_rn(__fsub_rn(t_hi, c_hi), __fsub_rn(t_lo, c_lo));
    const float corr = __fmul_rn(r, rcp_approx(__fmul_rn(3.0f, s_hi)));
    y = __fsub_rn(y0, corr);
    e = __fsub_rn(__fsub_rn(y0, y), corr);
    const uint32_t yb = __float_as_uint(y);
    const float ulp = __uint_as_float((yb & 0x7f800000u) - (23u << 23));
    const float gap = (e < 0.0f && (yb & 0x007fffffu) == 0u) ? 0.5f * ulp : ulp;
    return fabsf(e) > gap * (0.5f - 2.44140625e-4f) ||
           !(hf >= 9.5367431640625e-07f && hf <= 1048576.0f);
}

__device__ __forceinline__ float cbrt_sq_settle(float hf, float y, float e)
{
    if (!(hf >= 9.5367431640625e-07f && hf <= 1048576.0f))
        return cbrt_sq_wide(hf);
    return cbrt_sq_fix(hf, y, e);
}

// True when min(v, RN(sqrt(g*hf))) is not v, i.e. v*v > g*hf exactly
// (lexicographic comparison of the exact products as float pairs).
__device__ __forceinline__ bool vcr_caps(float v, float g, float hf)
{
    const float v2 = __fmul_rn(v, v), v2l = __fmaf_rn(v, v, -v2);
    const float p = __fmul_rn(g, hf), pl = __fmaf_rn(g, hf, -p);
    return v2 > p || (v2 == p && v2l > pl);
}

// RN_float(cbrt(hf*hf)) for hf > 0.
__device__ __forceinline__ float cbrt_sq_rn(float hf)
{
    // The float-pair estimate below is accurate to ~2^-39 relative for
    // hf in [2^-20, 2^20]; outside that, use the double cube root.
    if (!(hf >= 9.5367431640625e-07f && hf <= 1048576.0f))
        return cbrt_sq_wide(hf);
    float y0 = ex2_approx(__fmul_rn(lg2_approx(hf), 0.666666687f));
    float c_hi = __fmul_rn(hf, hf);
    float c_lo = __fmaf_rn(hf, hf, -c_hi);
    float s_hi = __fmul_rn(y0, y0);
    float s_lo = __fmaf_rn(y0, y0, -s_hi);
    float t_hi = __fmul_rn(s_hi, y0);
    float t_lo = __fmaf_rn(s_hi, y0, -t_hi);
    t_lo = __fmaf_rn(s_lo, y0, t_lo);
    // y0^3 - hf^2; t_hi - c_hi is exact (the operands are within a factor 2)
    float r = __fadd_rn(__fsub_rn(t_hi, c_hi), __fsub_rn(t_lo, c_lo));
    float corr = __fmul_rn(r, rcp_approx(__fmul_rn(3.0f, s_hi)));
    float y = __fsub_rn(y0, corr);
    // y0 - corr == y + e exactly (Fast2Sum, |y0| >> |corr|)
    float e = __fsub_rn(__fsub_rn(y0, y), corr);
    uint32_t yb = __float_as_uint(y);
    float ulp = __uint_as_float((yb & 0x7f800000u) - (23u << 23));
    // half of the gap to the neighbour on e's side, less a 2^-12 ulp margin
    float gap = (e < 0.0f && (yb & 0x007fffffu) == 0u) ? 0.5f * ulp : ulp;
    if (fabsf(e) > gap * (0.5f - 2.44140625e-4f))
        return cbrt_sq_fix(hf, y, e);
    return y;
}

static __device__ __noinline__ float sqrt_prod_wide(float g, float hf)
{
    return (float)__dsqrt_rn((double)g * (double)hf);
}

// RN(sqrt(p)) for the exact product p = g*hf (48 bits, as (double)g*(double)hf
// is), in float arithmetic: s = RN(sqrt(RN(p))) is within an ulp of the
// answer; the residual p - s^2, taken exactly from float pairs, gives the
// correction c = (p - s^2)/(2s), and RN(s + c) is decided by the rounding
// error of s + c unless it lies within 2^-12 ulp of a midpoint, where the
// double square root decides.
__device__ __forceinline__ float sqrt_prod_rn(float g, float hf)
{
    const float p = __fmul_rn(g, hf), pl = __fmaf_rn(g, hf, -p);
    const float s = __fsqrt_rn(p);
    const float s2 = __fmul_rn(s, s), s2l = __fmaf_rn(s, s, -s2);
    // p - s2 is exact (the operands are within a factor 2)
    const float r = __fadd_rn(__fsub_rn(__fsub_rn(p, s2), s2l), pl);
    const float c = __fmul_rn(r, rcp_approx(__fmul_rn(2.0f, s)));
    const float y = __fadd_rn(s, c);
    const float e = __fsub_rn(c, __fsub_rn(y, s));   // s + c == y + e exactly
    const uint32_t yb = __float_as_uint(y);
    const float ulp = __uint_as_float((yb & 0x7f800000u) - (23u << 23));
    const float gap = (e < 0.0f && (yb & 0x007fffffu) == 0u) ? 0.5f * ulp : ulp;
    if (fabsf(e) > gap * (0.5f - 2.44140625e-4f) || !(p >= 1.1754944e-38f))
        return sqrt_prod_wide(g, hf);
    return y;
}

// min(v, RN(sqrt(g*hf))) with g*hf taken exactly (as (double)g*(double)hf is).
// v > RN(sqrt(p)) implies v*v > p, and v*v > p implies RN(sqrt(p)) <= v, so
// the capped value is needed exactly when v*v > p. A float test with a 2^-20
// margin settles most faces; the exact float-pair comparison the rest.
__device__ __forceinline__ float min_vcr_rn(float v, float g, float hf)
{
    const float v2 = __fmul_rn(v, v);
    const float p = __fmul_rn(g, hf);
    if (v2 < p * 0.99999905f)
        return v;
    const float v2l = __fmaf_rn(v, v, -v2);
    const float pl = __fmaf_rn(g, hf, -p);
    const bool above = v2 > p || (v2 == p && v2l > pl);
    return above ? sqrt_prod_rn(g, hf) : v;
}

// True when RN(sqrt(g*h)) cannot exceed vmax (vmax >= 0): g*h <= vmax^2,
// tested with a 2^-20 margin so the float products' rounding cannot matter.
__device__ __forceinline__ bool vcr_at_most(float vmax, float g, float h)
{
    return __fmul_rn(g, h) * 1.00000095f < __fmul_rn(vmax, vmax);
}

}  // namespace fcab
