// Two FP32 lanes in one 64-bit register pair, operated on by the sm_100a
// packed instructions add/sub/mul/fma.rn.f32x2. Each packed instruction
// rounds both halves exactly as the scalar .rn instruction would, so a
// computation written on pairs gives the same bits as the same computation on
// each half, provided no packed product feeds a packed sum (see mul2_sep). A packed
// instruction takes one issue slot for two operations; the FMA pipe still
// spends a cycle on each half. Comparisons, selects, min/max and the MUFU
// approximations have no packed form and run per half.
#pragma once

#include <cstdint>

#include "wca_math.cuh"

namespace fcab {

struct f2 {
    unsigned long long u;
};

__device__ __forceinline__ f2 mk2(float a, float b)
{
    f2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r.u) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ f2 bc2(float a) { return mk2(a, a); }
__device__ __forceinline__ void sp2(f2 v, float &a, float &b)
{
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v.u));
}
__device__ __forceinline__ float lo2(f2 v)
{
    float a, b;
    sp2(v, a, b);
    return a;
}
__device__ __forceinline__ float hi2(f2 v)
{
    float a, b;
    sp2(v, a, b);
    return b;
}

__device__ __forceinline__ f2 add2(f2 a, f2 b)
{
    f2 r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r.u) : "l"(a.u), "l"(b.u));
    return r;
}
__device__ __forceinline__ f2 sub2(f2 a, f2 b)
{
    f2 r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r.u) : "l"(a.u), "l"(b.u));
    return r;
}
__device__ __forceinline__ f2 mul2(f2 a, f2 b)
{
    f2 r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r.u) : "l"(a.u), "l"(b.u));
    return r;
}
// RN(a*b) per half, as two scalar products: ptxas (CUDA 12.9) contracts a
// mul.rn.f32x2 whose result feeds an add.rn.f32x2 or sub.rn.f32x2 into one
// fused multiply-add, even with --fmad=false, and folds fma.rn.f32x2 with a
// -0 addend back into that product; scalar mul.rn is never contracted. Use
// this wherever a product is later summed and both roundings must happen.
__device__ __forceinline__ f2 mul2_sep(f2 a, f2 b)
{
    return mk2(__fmul_rn(lo2(a), lo2(b)), __fmul_rn(hi2(a), hi2(b)));
}
// a*b + c with one rounding
__device__ __forceinline__ f2 fma2(f2 a, f2 b, f2 c)
{
    f2 r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r.u) : "l"(a.u), "l"(b.u), "l"(c.u));
    return r;
}

// Per-half operations.
__device__ __forceinline__ f2 max2(f2 a, f2 b)
{
    return mk2(fmaxf(lo2(a), lo2(b)), fmaxf(hi2(a), hi2(b)));
}
__device__ __forceinline__ f2 min2(f2 a, f2 b)
{
    return mk2(fminf(lo2(a), lo2(b)), fminf(hi2(a), hi2(b)));
}
// -a per half, as (-0) - a: exact for every number and both zeros (one
// packed add instead of two integer operations)
__device__ __forceinline__ f2 neg2(f2 a)
{
    f2 r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r.u) : "l"(0x8000000080000000ull), "l"(a.u));
    return r;
}
__device__ __forceinline__ f2 abs2(f2 a)
{
    f2 r;
    r.u = a.u & 0x7fffffff7fffffffull;
    return r;
}
// magnitude of a with the sign of s, per half
__device__ __forceinline__ f2 copysign2(f2 a, f2 s)
{
    f2 r;
    r.u = (a.u & 0x7fffffff7fffffffull) | (s.u & 0x8000000080000000ull);
    return r;
}
__device__ __forceinline__ f2 sel2(bool p0, bool p1, f2 a, f2 b)
{
    return mk2(p0 ? lo2(a) : lo2(b), p1 ? hi2(a) : hi2(b));
}
__device__ __forceinline__ f2 lg2_2(f2 a) { return mk2(lg2_approx(lo2(a)), lg2_approx(hi2(a))); }
__device__ __forceinline__ f2 ex2_2(f2 a) { return mk2(ex2_approx(lo2(a)), ex2_approx(hi2(a))); }
__device__ __forceinline__ f2 rcp_2(f2 a) { return mk2(rcp_approx(lo2(a)), rcp_approx(hi2(a))); }
__device__ __forceinline__ f2 rsqrt_2(f2 a)
{
    return mk2(rsqrt_approx(lo2(a)), rsqrt_approx(hi2(a)));
}

// Sets / reads half j.
__device__ __forceinline__ void put2(f2 &v, int j, float x)
{
    v = j == 0 ? mk2(x, hi2(v)) : mk2(lo2(v), x);
}
__device__ __forceinline__ float get2(f2 v, int j) { return j == 0 ? lo2(v) : hi2(v); }

// Pair of this lane's right neighbours (b, next lane's a) and left
// neighbours (previous lane's b, a), by one shuffle each.
__device__ __forceinline__ f2 right2(f2 v)
{
    return mk2(hi2(v), __shfl_down_sync(0xffffffffu, lo2(v), 1));
}
__device__ __forceinline__ f2 left2(f2 v)
{
    return mk2(__shfl_up_sync(0xffffffffu, hi2(v), 1), lo2(v));
}

// ---- correctly rounded operations on pairs (normal-range operands) -------

// RN(a/b) per half given rb = RN(1/b) (Markstein; see div_mk).
__device__ __forceinline__ f2 div2_mk(f2 a, f2 b, f2 rb)
{
    const f2 q = mul2(a, rb);
    const f2 r = fma2(neg2(q), b, a);
    return fma2(r, rb, q);
}
// RN(1/x) per half (see rcp_nr).
__device__ __forceinline__ f2 rcp2_nr(f2 x)
{
    const f2 y = rcp_2(x);
    const f2 e = fma2(neg2(x), y, bc2(1.0f));
    return fma2(e, y, y);
}
// RN(sqrt(x)) per half, x normal and positive (see sqrt_nr).
__device__ __forceinline__ f2 sqrt2_nr(f2 x)
{
    const f2 y = rsqrt_2(x);
    const f2 s = mul2(x, y);
    const f2 h = mul2(bc2(0.5f), y);
    const f2 r = fma2(neg2(s), s, x);
    return fma2(r, h, s);
}

// hf^(2/3) = RN(cbrt(hf*hf)) per half, without the exactness fix-up: the
// cube root u of hf by one Newton step on a log2/exp2 estimate u0
// (u = u0 - (u0^3 - hf)/(3 u0^2), the residual taken exactly by fused
// multiply-adds), then u^2 as the float pair s_hi + t, t = s_lo - 2 u0 corr,
// rounded to y with its rounding error e (Fast2Sum). The value y + e is
// within about 2^-40 relative of cbrt(hf^2) for hf in [2^-20, 2^20].
// `unsure` (per half) is set when that is not enough to decide the rounding:
// |e| within 2^-11 of half an ulp of y (tested as fma(e, 1 + 2^-11, y) != y,
// which also covers the halved gap below a power of two), or hf outside
// [2^-20, 2^20]; the caller then evaluates those halves exactly.
__device__ __forceinline__ f2 cbrt_sq2(f2 hf, bool &unsure0, bool &unsure1)
{
    const f2 l = lg2_2(hf);
    const f2 u0 = ex2_2(mul2(l, bc2(0.333333343f)));
    const f2 s_hi = mul2_sep(u0, u0);
    const f2 s_lo = fma2(u0, u0, neg2(s_hi));
    const f2 r1 = fma2(s_hi, u0, neg2(hf));
    const f2 r = fma2(s_lo, u0, r1);                        // u0^3 - hf
    const f2 c2 = mul2(r, rcp_2(mul2(bc2(1.5f), s_hi)));    // 2 (u0 - u)
    const f2 t = fma2(u0, neg2(c2), s_lo);
    const f2 y = add2(s_hi, t);
    const f2 e = add2(sub2(s_hi, y), t);
    const f2 chk = fma2(e, bc2(1.00048828125f), y);
    float l0, l1, y0, y1, k0, k1;
    sp2(l, l0, l1);
    sp2(y, y0, y1);
    sp2(chk, k0, k1);
    unsure0 = k0 != y0 || !(fabsf(l0) <= 20.0f);
    unsure1 = k1 != y1 || !(fabsf(l1) <= 20.0f);
    return y;
}

}  // namespace fcab
