// Device formulas of the WCA rule, re-derived from FloodCA
// src/kernels/physics.h for the sm_100a kernels. The expression order of
// every rounded operation follows the reference so that the float build
// (MATH_EXACT) and the double build give the reference's values; MATH_FAST
// replaces cbrt, sqrt and divisions with hardware approximations.
#pragma once

#include "wca_math.cuh"

namespace fcab {

enum : uint8_t { M_LAND = 0, M_SEA = 1, M_WALL = 2 };
enum { MATH_EXACT = 0, MATH_FAST = 1 };

// Per-step constants shared by every face of one step.
template <typename T>
struct StepK {
    T dx, A, g, tau_h, tau_l, z_sea, S_bnd;
    T w;          // face width: dx (K=4) or (sqrt2-1)dx (K=8), physics.h:37-43
    T d_diag;     // sqrt2*dx, physics.h:45-48
    T dt;         // this step's dt
    T den;        // (2K)*dt, denominator of the volume cap
    T rden;       // RN(1/den), used to skip the cap division when far from capping
    T rdx, rdd;   // 1/dx, 1/d_diag (fast mode)
    T alpha_dx;   // alpha*dx
    T inv_A;      // 1/A (fast mode)
};

// --- hf^(2/3), sqrt and Manning velocity in each precision / mode ---------

template <typename T, int MATH>
struct Mth;

template <>
struct Mth<float, MATH_EXACT> {
    // a/b given rb = RN(1/b): Markstein's correction, exact for normal operands
    static __device__ __forceinline__ float div_c(float a, float b, float rb)
    {
        return div_mk(a, b, rb);
    }
    static __device__ __forceinline__ float rcp_bf(float a) { return rcp_nr(a); }
    static __device__ __forceinline__ float sqrt_bf(float a) { return sqrt_nr(a); }
    static __device__ __forceinline__ bool cbrt_try(float x, float &y, float &e)
    {
        return cbrt_sq_try(x, y, e);
    }
    static __device__ __forceinline__ float cbrt_settle(float x, float y, float e)
    {
        return cbrt_sq_settle(x, y, e);
    }
    static __device__ __forceinline__ bool caps(float v, float g, float h) { return vcr_caps(v, g, h); }
    static __device__ __forceinline__ float vcr(float g, float h) { return sqrt_prod_rn(g, h); }
    static __device__ __forceinline__ float cbrt_sq(float x) { return cbrt_sq_rn(x); }
    static __device__ __forceinline__ float sqrt_(float x) { return __fsqrt_rn(x); }
    static __device__ __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }
    static __device__ __forceinline__ float rcp(float a) { return __frcp_rn(a); }
    static __device__ __forceinline__ float min_vcr(float v, float g, float h)
    {
        return min_vcr_rn(v, g, h);
    }
    static __device__ __forceinline__ bool vcr_le(float vmax, float g, float h)
    {
        return vcr_at_most(vmax, g, h);
    }
};

template <>
struct Mth<float, MATH_FAST> {
    static __device__ __forceinline__ float div_c(float a, float, float rb) { return a * rb; }
    static __device__ __forceinline__ float rcp_bf(float a) { return rcp_approx(a); }
    static __device__ __forceinline__ float sqrt_bf(float a) { return a * rsqrt_approx(a); }
    static __device__ __forceinline__ bool cbrt_try(float x, float &y, float &e)
    {
        y = ex2_approx(lg2_approx(x) * 0.666666687f);
        e = 0.0f;
        return false;
    }
    static __device__ __forceinline__ float cbrt_settle(float, float y, float) { return y; }
    static __device__ __forceinline__ bool caps(float v, float g, float h) { return v * v > g * h; }
    static __device__ __forceinline__ float vcr(float g, float h)
    {
        const float p = g * h;
        return p * rsqrt_approx(p);
    }
    static __device__ __forceinline__ float cbrt_sq(float x)
    {
        return ex2_approx(lg2_approx(x) * 0.666666687f);
    }
    static __device__ __forceinline__ float sqrt_(float x) { return x * rsqrt_approx(x); }
    static __device__ __forceinline__ float div(float a, float b) { return a * rcp_approx(b); }
    static __device__ __forceinline__ float rcp(float a) { return rcp_approx(a); }
    static __device__ __forceinline__ float min_vcr(float v, float g, float h)
    {
        float p = g * h;
        float vcr = p * rsqrt_approx(p);
        return v > vcr ? vcr : v;
    }
    static __device__ __forceinline__ bool vcr_le(float vmax, float g, float h)
    {
        return g * h * 1.0001f <= vmax * vmax;
    }
};

template <int MATH>
struct Mth<double, MATH> {
    static __device__ __forceinline__ double div_c(double a, double b, double)
    {
        return __ddiv_rn(a, b);
    }
    static __device__ __forceinline__ double rcp_bf(double a) { return __drcp_rn(a); }
    static __device__ __forceinline__ double sqrt_bf(double a) { return __dsqrt_rn(a); }
    static __device__ __forceinline__ bool cbrt_try(double x, double &y, double &e)
    {
        y = cbrt(x * x);
        e = 0.0;
        return false;
    }
    static __device__ __forceinline__ double cbrt_settle(double, double y, double) { return y; }
    static __device__ __forceinline__ bool caps(double v, double g, double h)
    {
        return v > __dsqrt_rn(g * h);
    }
    static __device__ __forceinline__ double vcr(double g, double h) { return __dsqrt_rn(g * h); }
    static __device__ __forceinline__ double cbrt_sq(double x) { return cbrt(x * x); }
    static __device__ __forceinline__ double sqrt_(double x) { return __dsqrt_rn(x); }
    static __device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
    static __device__ __forceinline__ double rcp(double a) { return __drcp_rn(a); }
    static __device__ __forceinline__ double min_vcr(double v, double g, double h)
    {
        double vcr = __dsqrt_rn(g * h);
        return v > vcr ? vcr : v;
    }
    static __device__ __forceinline__ bool vcr_le(double vmax, double g, double h)
    {
        return __dsqrt_rn(g * h) <= vmax;
    }
};

// --- face discharge (physics.h:51-125) -------------------------------------

// Signed discharge a->b across a face of centre distance d (dx, or the
// diagonal distance). rd = 1/d for the fast mode. cap is set when the volume
// cap |dL|*A/(2K*dt) binds.
template <typename T, int MATH>
__device__ __forceinline__ T face_q(T za, T ha, T na, uint32_t ma, T zb, T hb, T nb, uint32_t mb,
                                    T d, T rd, const StepK<T> &k, int &cap)
{
    using M = Mth<T, MATH>;
    cap = 0;
    if (ma == M_WALL || mb == M_WALL)
        return T(0);
    const bool sa = ma == M_SEA, sb = mb == M_SEA;
    T zea = sa ? k.z_sea : za;
    T zeb = sb ? k.z_sea : zb;
    T la = zea + (sa ? T(0) : ha);
    T lb = zeb + (sb ? T(0) : hb);
    T dL = la - lb;
    T adL = dL < T(0) ? -dL : dL;
    if (adL < k.tau_l)
        return T(0);
    T hf = (la > lb ? la : lb) - (zea > zeb ? zea : zeb);
    if (hf < k.tau_h)
        return T(0);
    if (dL > T(0) ? sa : sb)
        return T(0);
    T nf = sa ? nb : (sb ? na : T(0.5) * (na + nb));
    if (nf < T(1e-12))
        nf = T(1e-12);
    T S = MATH == MATH_EXACT ? M::div(adL, d) : adL * rd;
    T v = M::rcp(nf) * M::cbrt_sq(hf) * M::sqrt_(S);
    v = M::min_vcr(v, k.g, hf);
    T Qm = v * hf * k.w;
    T num = adL * k.A;
    // Cap test: skip the exact division when the estimate num*rden is clearly
    // above Qm (relative error of the estimate is below 2^-22).
    if (MATH == MATH_EXACT) {
        if (!(num * k.rden > Qm * T(1.0000005))) {
            T Qc = M::div(num, k.den);
            if (Qc < Qm) {
                cap = 1;
                Qm = Qc;
            }
        }
    } else {
        T Qc = num * k.rden;
        if (Qc < Qm) {
            cap = 1;
            Qm = Qc;
        }
    }
    return dL > T(0) ? Qm : -Qm;
}

// Discharge of NF independent faces at once (the same formula as face_q),
// arranged in phases so that each phase is one branch-free block over all
// faces: the compiler interleaves the faces' dependency chains. Faces that
// carry no flow (walls, |dL| < tau_l, hf < tau_h, upwind SEA) are evaluated
// on safe operands and zeroed at the end. The rare exact-rounding
// settlements (cube root near a midpoint, critical-velocity cap) run after
// their phase in per-lane blocks.
template <typename T, int MATH, bool LANDONLY, int NF>
__device__ __forceinline__ void faces_q(const T (&za)[NF], const T (&ha)[NF], const T (&na)[NF],
                                        const uint32_t (&ma)[NF], const T (&zb)[NF],
                                        const T (&hb)[NF], const T (&nb)[NF],
                                        const uint32_t (&mb)[NF], const T (&d)[NF],
                                        const T (&rd)[NF], const StepK<T> &k, T (&Q)[NF],
                                        unsigned (&cap)[NF])
{
    using M = Mth<T, MATH>;
    // sL: signed level difference of a live face, 0 for a face that carries
    // no flow (so no boolean state crosses the phases)
    T hf[NF], sL[NF], nf[NF], cb[NF], ce[NF];
    unsigned settle = 0u;
#pragma unroll
    for (int f = 0; f < NF; f++) {
        T zea, zeb, la, lb, n;
        bool dd = false;
        if constexpr (LANDONLY) {
            zea = za[f];
            zeb = zb[f];
            la = za[f] + ha[f];
            lb = zb[f] + hb[f];
            n = T(0.5) * (na[f] + nb[f]);
        } else {
            const bool sa = ma[f] == M_SEA, sb = mb[f] == M_SEA;
            dd = ma[f] == M_WALL || mb[f] == M_WALL;
            zea = sa ? k.z_sea : za[f];
            zeb = sb ? k.z_sea : zb[f];
            la = zea + (sa ? T(0) : ha[f]);
            lb = zeb + (sb ? T(0) : hb[f]);
            n = sa ? nb[f] : (sb ? na[f] : T(0.5) * (na[f] + nb[f]));
            dd = dd || ((la - lb) > T(0) ? sa : sb);
        }
        const T dL = la - lb;
        const T h = (la > lb ? la : lb) - (zea > zeb ? zea : zeb);
        dd = dd || fabs(dL) < k.tau_l || h < k.tau_h;
        // a dead face's hf is replaced so the cube root stays on its fast
        // path; its other operands may produce NaN, which the final select drops
        hf[f] = dd ? T(1) : h;
        sL[f] = dd ? T(0) : dL;
        nf[f] = n < T(1e-12) ? T(1e-12) : n;
        if (M::cbrt_try(hf[f], cb[f], ce[f]))
            settle |= 1u << f;
    }
    if (settle) {
#pragma unroll
        for (int f = 0; f < NF; f++)
            if (settle & (1u << f))
                cb[f] = M::cbrt_settle(hf[f], cb[f], ce[f]);
    }
    T v[NF];
    unsigned capv = 0u;
#pragma unroll
    for (int f = 0; f < NF; f++) {
        const T S = M::div_c(fabs(sL[f]), d[f], rd[f]);
        v[f] = M::rcp_bf(nf[f]) * cb[f] * M::sqrt_bf(S);
        if (M::caps(v[f], k.g, hf[f]))
            capv |= 1u << f;
    }
    if (capv) {
#pragma unroll
        for (int f = 0; f < NF; f++)
            if (capv & (1u << f))
                v[f] = M::vcr(k.g, hf[f]);
    }
#pragma unroll
    for (int f = 0; f < NF; f++) {
        T Qm = v[f] * hf[f] * k.w;
        const T Qc = M::div_c(fabs(sL[f]) * k.A, k.den, k.rden);
        const bool c = Qc < Qm;
        Qm = c ? Qc : Qm;
        const bool live = sL[f] != T(0);
        cap[f] = (live && c) ? 1u : 0u;
        Q[f] = live ? copysign(Qm, sL[f]) : T(0);
    }
}

// Upper bound of cell_velocity (relative error of the float approximations
// below 1e-5): max(min(h^(2/3) sqrt(S) / n, sqrt(g h)), 1e-6) * (1 + 1e-4).
template <typename T>
__device__ __forceinline__ T cell_velocity_bound(T h, T n, T S, const StepK<T> &k)
{
    if constexpr (sizeof(T) == 4) {
        const float nn = n < 1e-12f ? 1e-12f : n;
        const float cb = ex2_approx(lg2_approx(h) * 0.666666687f);
        const float sq = S > 0.0f ? S * rsqrt_approx(S) : 0.0f;
        float v = rcp_approx(nn) * cb * sq;
        const float p = k.g * h;
        const float vc = p * rsqrt_approx(p);
        v = v < vc ? v : vc;
        v = v < 1e-6f ? 1e-6f : v;
        return v * 1.0001f;
    } else {
        return T(1e300);   // no bound: the FP64 kernels evaluate every candidate
    }
}

// Limiter without branches (physics.h:127-134): hold/out when the outflow
// volume exceeds the held volume, else 1.
template <typename T, int MATH>
__device__ __forceinline__ T limiter_bf(T out_vol, T h, T A)
{
    using M = Mth<T, MATH>;
    const T hold = h * A;
    const bool lim = out_vol > hold && out_vol > T(0);
    const T o = lim ? out_vol : T(1);
    const T q = M::div_c(hold, o, M::rcp_bf(o));
    return lim ? q : T(1);
}

// Open-edge discharge to the virtual neighbour z - S_bnd*dx, h = 0, same n,
// distance dx, clipped at zero (FloodCA src/common/model.c:166-177).
template <typename T, int MATH>
__device__ __forceinline__ T open_q(T z, T h, T n, uint32_t m, const StepK<T> &k, int &cap)
{
    T Q = face_q<T, MATH>(z, h, n, m, z - k.S_bnd * k.dx, T(0), n, M_LAND, k.dx, k.rdx, k, cap);
    return Q < T(0) ? T(0) : Q;
}

// Sum of k copies of q in the order of the reference's four open slots
// (model.c:235-236): the zero slots do not change the partial sums.
template <typename T>
__device__ __forceinline__ T open_sum(T q, int kcnt)
{
    T s = kcnt > 0 ? q : T(0);
    const T s2 = s + q;
    s = kcnt > 1 ? s2 : s;
    const T s3 = s + q;
    s = kcnt > 2 ? s3 : s;
    const T s4 = s + q;
    return kcnt > 3 ? s4 : s;
}

// Limiter (physics.h:127-134).
template <typename T, int MATH>
__device__ __forceinline__ T limiter_s(T out_vol, T h, T A)
{
    T hold = h * A;
    if (out_vol > hold && out_vol > T(0))
        return Mth<T, MATH>::div(hold, out_vol);
    return T(1);
}

// Velocity whose alpha*dx/v is the cell's stable step (physics.h:193-217),
// for a wet LAND cell (h >= tau_h); Smax is the largest surface slope.
template <typename T, int MATH>
__device__ __forceinline__ T cell_velocity(T h, T n, T Smax, const StepK<T> &k)
{
    using M = Mth<T, MATH>;
    if (n < T(1e-12))
        n = T(1e-12);
    if (Smax < T(0))
        Smax = T(0);
    T v = M::rcp(n) * M::cbrt_sq(h) * M::sqrt_(Smax);
    v = M::min_vcr(v, k.g, h);
    if (v < T(1e-6))
        v = T(1e-6);
    return v;
}

}  // namespace fcab
