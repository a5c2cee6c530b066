// Fused WCA step kernel for sm_100a.
//
// One launch = one step of FloodCA's fca_step (src/common/model.c:321-605)
// over the whole grid, with the next step's stable-dt reduction
// (model.c:111-156) fused in and all step control (dt clamp, event clamp,
// hyetograph integral, time advance; model.c:363-382, 600-601,
// src/common/rain.c:30-93) kept on the device, so the host never waits
// inside a run.
//
// Work decomposition: a warp streams down a vertical strip of 32*CPL columns
// (lane l holds CPL adjacent columns), one input row per iteration, through a
// register pipeline:
//   iteration i loads row i+1 (prefetch) and computes
//     A  x-face discharge of row i and y-face (and diagonal) discharge
//        between rows i-1 and i              (physics.h:51-125)
//     C  outflow sum and limiter s of row i-1  (model.c:489-502)
//     D  limiter-scaled net inflow, rain, clamp, hmax/tmax of row i-2
//        (model.c:511-597); the row is written if it is an output row
//     E  the next step's per-cell stable velocity of row i-3 from the new
//        depths of rows i-4..i-2 (physics.h:158-217)
// Horizontal neighbours come from the adjacent lane by warp shuffle. A strip
// overlaps its neighbours by HL columns on each side (3 halo columns are
// needed: E at column c needs new depth at c+-1, which needs s at c+-2,
// which needs fluxes reaching c+-3), so only its middle OW columns are
// written. Every warp owns a contiguous, balanced range of (strip, row)
// pairs; the vertical halo costs 6 pipeline iterations per segment.
//
// The minimum over cells of alpha*dx/v equals alpha*dx / max(v) (division by
// a positive number rounds monotonically), so warps reduce max(v) and
// publish it with one atomicMax on the float bit pattern. The last CTA to
// finish prepares the next step's control block.
#pragma once

#include <cuda.h>

#include "wca_physics.cuh"

namespace fcab {

constexpr int PADR = 8;   // padded rows above and below the grid (the pair sweep
                          // starts up to six rows above a segment)
constexpr int PADC = 4;   // padded columns left of the grid
constexpr int NSLOT = 32; // accumulator slots (spread the atomics)
constexpr double PAD_Z = 1e30;   // padding elevation of all-LAND grids

template <int CPL>
struct Geom {
    static constexpr int HL = CPL == 1 ? 3 : 4;     // halo columns each side
    static constexpr int SW = 32 * CPL;             // strip width (columns)
    static constexpr int OW = SW - 2 * HL;          // output columns per strip
};

// Device view of the padded grid. Element (r, c) of the nrows x ncols grid is
// at index (r + PADR) * pitch + (c + PADC); padding cells are WALL with zero
// z, h and n.
template <typename T>
struct GridD {
    const T *z, *n, *cr;        // cr: per-cell C*Rday, or nullptr
    const uint8_t *m;
    T *h0, *h1, *hmax, *tmax;
    long long pitch;
    int nr, nc;
    int r_lo, r_hi;             // rows of real cells: [0, nr), or with a slab's halo rows
    // row-tile tensor maps of z, n, h0, h1 (device memory) for the TMA row
    // source of the FP32 pair sweep, or nullptr (plain loads)
    const CUtensorMap *tmap = nullptr;
};

// Uniform run constants.
template <typename T>
struct RunK {
    StepK<T> k;                 // dt-independent members filled
    T dt_max, dt_min, cr_uniform;
    int K, U, open, edge_n, edge_s, edge_w, edge_e;
    int inflow_r, inflow_c;     // -1: none
    int has_sea;
};

// Fraction of a step's velocity maximum that seeds the next step's dt
// pruning.
#ifndef FCAB_VSEED_FRAC
#define FCAB_VSEED_FRAC 0.9
#endif

// Host-visible control block; one per run, in device memory.
struct Ctl {
    // prepared for the next step by the previous step's last CTA
    double t, dt, F, tmax_val, inflow_dh, t_next, dt_base;
    int step, hit, active, h_cur, want_v, done, pause, force_day;
    int err, n_force_days;
    int fin_pending;            // slab runs: 1 after a step, 2 after the first velocity pass
    int inflow_off;             // 1: the inflow cell is not LAND (no inflow volume)
    long long dt_min_hits;
    unsigned long long vmax_bits;
    unsigned int ctas_done;
    unsigned int launches;
    double window_end;          // > 0: pause once t reaches it (batched ensembles)
    double V_in;                // inflow volume added by the steps taken
    double V_in_step;           // inflow volume of the prepared step
    // velocity seed of the next step's dt pruning (float or double bits, 0:
    // none) and the deferred-dt handshake with the full velocity pass
    unsigned long long vseed_bits;
    int need_v;                 // the step's pruned maximum fell below the seed
    int pause_carry;            // progress pause decided before the deferral
    long long full_passes;      // deferred dts completed by the full pass
    double accd[4][NSLOT];      // V_rain, clamp, V_sea, V_bnd (double accumulation)
    float accf[4][NSLOT];       // same, FP32 accumulation
    unsigned long long cap[NSLOT];
};

// Event and forcing parameters for the device-side step control.
struct TimeCfg {
    double T_sim, out_every, D_h, phi, rain_end;
    double inflow_peak, inflow_t_peak, inflow_t_end;
    double alpha_dx_d;
    int hyeto, max_steps, U, time_f32;
    int n_force_days, progress_every, inflow_ok, prec_f64;
    int vseed_on;               // seed the dt pruning (a missed seed needs the full pass)
    int split;                  // slab of a row-split domain: the step control waits for
                                // the velocity maximum reduced over all slabs
    int tail_vpass;             // the step kernel itself tail-launches the full velocity
                                // pass when its seed missed (else the launcher adds it)
};

// --------------------------------------------------------------------------
// Step control (device, one thread): FloodCA src/common/rain.c:8-93 and the
// loop of src/common/model.c:607-643.

__device__ __forceinline__ double tri_f(double t, double T, double tp)
{
    if (t < 0.0 || t >= T || T <= 0.0)
        return 0.0;
    if (t < tp)
        return tp <= 0.0 ? 0.0 : (2.0 / T) * (t / tp);
    return T - tp <= 0.0 ? 0.0 : (2.0 / T) * ((T - t) / (T - tp));
}

__device__ inline double hyeto_integral(const TimeCfg &c, double t, double dt)
{
    if (dt <= 0.0)
        return 0.0;
    double t1 = t + dt;
    if (c.hyeto == 1)
        return dt / 86400.0;
    double T = c.D_h * 3600.0, tp = c.phi * T, sum = 0.0, a;
    if (t1 <= 0.0 || t >= T)
        return 0.0;
    if (t < 0.0)
        t = 0.0;
    if (t1 > T)
        t1 = T;
    a = t;
    for (int guard = 0; a < t1 - 1e-15 && guard < 4; guard++) {
        double b = (a < tp && t1 > tp) ? tp : t1;
        sum += 0.5 * (tri_f(a, T, tp) + tri_f(b, T, tp)) * (b - a);
        a = b;
    }
    return sum;
}

__device__ inline double next_event(const TimeCfg &c, double t)
{
    double t_next = c.T_sim;
    double t_day = (floor(t / 86400.0) + 1.0) * 86400.0;
    if (t_day - t < 1e-9)
        t_day += 86400.0;
    if (t_day < t_next)
        t_next = t_day;
    if (c.out_every > 0.0) {
        double t_out = (floor(t / c.out_every) + 1.0) * c.out_every;
        if (t_out - t < 1e-9)
            t_out += c.out_every;
        if (t_out < t_next)
            t_next = t_out;
    }
    if (c.rain_end > 0.0 && c.rain_end - t >= 1e-9 && c.rain_end < t_next)
        t_next = c.rain_end;
    return t_next;
}

__device__ inline double inflow_rate(const TimeCfg &c, double t)
{
    if (t <= 0.0 || t >= c.inflow_t_end)
        return 0.0;
    if (t <= c.inflow_t_peak)
        return c.inflow_t_peak > 0.0 ? c.inflow_peak * (t / c.inflow_t_peak) : c.inflow_peak;
    return c.inflow_t_end > c.inflow_t_peak
               ? c.inflow_peak * ((c.inflow_t_end - t) / (c.inflow_t_end - c.inflow_t_peak))
               : 0.0;
}

__device__ inline double inflow_volume(const TimeCfg &c, double t, double dt)
{
    if (!c.inflow_ok || dt <= 0.0)
        return 0.0;
    double t1 = t + dt, a, sum = 0.0;
    if (t < 0.0)
        t = 0.0;
    if (t1 > c.inflow_t_end)
        t1 = c.inflow_t_end;
    a = t;
    for (int guard = 0; a < t1 && guard < 4; guard++) {
        double b = (a < c.inflow_t_peak && t1 > c.inflow_t_peak) ? c.inflow_t_peak : t1;
        sum += 0.5 * (inflow_rate(c, a) + inflow_rate(c, b)) * (b - a);
        a = b;
    }
    return sum;
}

// Prepares ctl for the step after the one just taken (after_step) or for
// the first step. Runs on one thread once every CTA's atomics are visible.
template <typename T>
__device__ void finalize(Ctl *c, const TimeCfg &tc, const RunK<T> &rk, bool after_step)
{
    double t = c->t;
    int step = c->step;
    if (after_step) {
        if (c->hit)
            t = c->t_next;
        else if (tc.time_f32)
            t = (double)((float)c->t + (float)c->dt);
        else
            t = c->t + c->dt;
        step += 1;
        c->V_in += c->V_in_step;
    }
    bool done = tc.max_steps > 0 ? step >= tc.max_steps : t >= tc.T_sim - 1e-15;
    int pause = 0;
    if (!done && tc.n_force_days > 0) {
        int d = t < 0.0 ? 0 : (int)floor(t / 86400.0);
        if (d >= tc.n_force_days)
            d = tc.n_force_days - 1;
        if (d != c->force_day)
            pause = 1;              // the host loads the day's Rday, then resumes
    }
    if (!done && after_step && tc.progress_every > 0 && step % tc.progress_every == 0)
        pause = 1;
    if (!done && c->pause_carry)
        pause = 1;                  // decided before a deferred dt
    if (!done && c->window_end > 0.0 && t >= c->window_end - 1e-9)
        pause = 1;                  // end of an output window
    T dt_base = (T)c->dt_base;
    if (!done && step % tc.U == 0) {
        T vmax;
        if (sizeof(T) == 4)
            vmax = (T)__uint_as_float((unsigned)c->vmax_bits);
        else
            vmax = (T)__longlong_as_double((long long)c->vmax_bits);
        T seed;
        if (sizeof(T) == 4)
            seed = (T)__uint_as_float((unsigned)c->vseed_bits);
        else
            seed = (T)__longlong_as_double((long long)c->vseed_bits);
        if (after_step && tc.vseed_on && vmax < seed) {
            c->full_passes += 1;
            // cells pruned against the seed may hold the maximum: keep the
            // time advance, defer dt to the full velocity pass (k_init_dt)
            c->t = t;
            c->step = step;
            c->pause_carry = pause;
            c->need_v = 1;
            c->active = 0;
            c->vmax_bits = 0ull;
            c->ctas_done = 0u;
            return;
        }
        // seed of the next dt computation: pruning against FCAB_VSEED_FRAC of this
        // step's maximum; a step whose maximum falls below it is redone
        // by the full pass
        if (tc.vseed_on) {
            const T sd = vmax * T(FCAB_VSEED_FRAC);
            if (sizeof(T) == 4)
                c->vseed_bits = (unsigned long long)__float_as_uint((float)sd);
            else
                c->vseed_bits = (unsigned long long)__double_as_longlong((double)sd);
        } else {
            c->vseed_bits = 0ull;
        }
        T dtm = rk.dt_max;
        if (vmax > T(0)) {
            T dta = rk.k.alpha_dx / vmax;
            if (dta < dtm)
                dtm = dta;
        }
        if (dtm < rk.dt_min) {
            dtm = rk.dt_min;
            c->dt_min_hits += 1;
        }
        if (dtm > rk.dt_max)
            dtm = rk.dt_max;
        dt_base = dtm;
    }
    T dt = dt_base;
    double t_next = 0.0;
    int hit = 0;
    double F = 0.0, V_in = 0.0;
    if (!done) {
        t_next = next_event(tc, t);
        double remain = t_next - t;
        if (remain <= (double)dt) {
            if (remain < 0.0)
                remain = 0.0;
            dt = (T)remain;
            hit = 1;
        }
        if (!(dt > T(0)))
            done = true;            // the reference loop stops advancing here
    }
    if (!done) {
        bool rain_on = tc.rain_end <= 0.0 || tc.rain_end - t >= 1e-9;
        F = rain_on ? hyeto_integral(tc, t, (double)dt) : 0.0;
        V_in = c->inflow_off ? 0.0 : inflow_volume(tc, t, (double)dt);
    }
    c->t = t;
    c->step = step;
    c->dt_base = (double)dt_base;
    c->dt = (double)dt;
    c->t_next = t_next;
    c->hit = hit;
    c->F = F;
    c->inflow_dh = (double)(T)(V_in / (double)rk.k.A);
    c->V_in_step = V_in;
    if (tc.time_f32)
        c->tmax_val = (double)((float)t + (float)dt);
    else
        c->tmax_val = t + (double)dt;
    c->want_v = (step + 1) % tc.U == 0;
    c->need_v = 0;
    c->pause_carry = 0;
    c->done = done ? 1 : 0;
    c->pause = pause;
    c->active = (!done && !pause) ? 1 : 0;
    c->vmax_bits = 0ull;
    c->ctas_done = 0u;
}

// --------------------------------------------------------------------------
// Row loads (vectorised by CPL).

template <typename T, int CPL>
struct VecIO;

template <int CPL>
struct VecIO<float, CPL> {
    static __device__ __forceinline__ void ld(float (&x)[CPL], const float *p)
    {
        if constexpr (CPL == 4) {
            float4 v = __ldg(reinterpret_cast<const float4 *>(p));
            x[0] = v.x; x[1] = v.y; x[2] = v.z; x[3] = v.w;
        } else if constexpr (CPL == 2) {
            float2 v = __ldg(reinterpret_cast<const float2 *>(p));
            x[0] = v.x; x[1] = v.y;
        } else {
            x[0] = __ldg(p);
        }
    }
    static __device__ __forceinline__ void ld_rw(float (&x)[CPL], const float *p)
    {
        if constexpr (CPL == 4) {
            float4 v = *reinterpret_cast<const float4 *>(p);
            x[0] = v.x; x[1] = v.y; x[2] = v.z; x[3] = v.w;
        } else if constexpr (CPL == 2) {
            float2 v = *reinterpret_cast<const float2 *>(p);
            x[0] = v.x; x[1] = v.y;
        } else {
            x[0] = *p;
        }
    }
    static __device__ __forceinline__ void st(float *p, const float (&x)[CPL])
    {
        if constexpr (CPL == 4)
            *reinterpret_cast<float4 *>(p) = make_float4(x[0], x[1], x[2], x[3]);
        else if constexpr (CPL == 2)
            *reinterpret_cast<float2 *>(p) = make_float2(x[0], x[1]);
        else
            *p = x[0];
    }
};

template <int CPL>
struct VecIO<double, CPL> {
    static __device__ __forceinline__ void ld(double (&x)[CPL], const double *p)
    {
#pragma unroll
        for (int j = 0; j < CPL; j += (CPL >= 2 ? 2 : 1)) {
            if constexpr (CPL >= 2) {
                double2 v = __ldg(reinterpret_cast<const double2 *>(p + j));
                x[j] = v.x;
                x[j + 1] = v.y;
            } else {
                x[j] = __ldg(p + j);
            }
        }
    }
    static __device__ __forceinline__ void ld_rw(double (&x)[CPL], const double *p)
    {
#pragma unroll
        for (int j = 0; j < CPL; j++)
            x[j] = p[j];
    }
    static __device__ __forceinline__ void st(double *p, const double (&x)[CPL])
    {
#pragma unroll
        for (int j = 0; j < CPL; j += (CPL >= 2 ? 2 : 1)) {
            if constexpr (CPL >= 2)
                *reinterpret_cast<double2 *>(p + j) = make_double2(x[j], x[j + 1]);
            else
                p[j] = x[j];
        }
    }
};

template <int CPL>
__device__ __forceinline__ void ld_mask(uint32_t (&m)[CPL], const uint8_t *p)
{
    if constexpr (CPL == 4) {
        uint32_t v = __ldg(reinterpret_cast<const unsigned int *>(p));
        m[0] = v & 0xffu; m[1] = (v >> 8) & 0xffu; m[2] = (v >> 16) & 0xffu; m[3] = v >> 24;
    } else if constexpr (CPL == 2) {
        uint32_t v = __ldg(reinterpret_cast<const unsigned short *>(p));
        m[0] = v & 0xffu; m[1] = v >> 8;
    } else {
        m[0] = __ldg(p);
    }
}

// Rows ahead of the current load that the sweep prefetches into L2.
constexpr int PF_ROWS = 3;

__device__ __forceinline__ void prefetch_l2(const void *p)
{
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

template <typename T, int CPL>
struct Row {
    T z[CPL], h[CPL], n[CPL];
    uint32_t m[CPL];
};

template <typename T, int CPL, bool LANDONLY>
__device__ __forceinline__ void load_row(Row<T, CPL> &R, const GridD<T> &g, const T *hin,
                                         long long off)
{
    VecIO<T, CPL>::ld(R.z, g.z + off);
    VecIO<T, CPL>::ld(R.h, hin + off);
    VecIO<T, CPL>::ld(R.n, g.n + off);
    if constexpr (LANDONLY) {
#pragma unroll
        for (int j = 0; j < CPL; j++)
            R.m[j] = M_LAND;
    } else {
        ld_mask<CPL>(R.m, g.m + off);
    }
}

template <typename T>
__device__ __forceinline__ T sh_dn(T v)
{
    return __shfl_down_sync(0xffffffffu, v, 1);
}
template <typename T>
__device__ __forceinline__ T sh_up(T v)
{
    return __shfl_up_sync(0xffffffffu, v, 1);
}

// Right / left neighbour of the lane's column j within a row held as CPL
// values per lane.
template <typename T, int CPL>
__device__ __forceinline__ T right_of(const T (&x)[CPL], int j, T nxt0)
{
    return j + 1 < CPL ? x[j + 1 < CPL ? j + 1 : 0] : nxt0;
}
template <typename T, int CPL>
__device__ __forceinline__ T left_of(const T (&x)[CPL], int j, T prv_last)
{
    return j > 0 ? x[j > 0 ? j - 1 : 0] : prv_last;
}

// Maximum over the warp of a non-negative value (positive floats order like
// their bit patterns, so the integer warp reduction applies).
template <typename T>
__device__ __forceinline__ T warp_max_nonneg(T v)
{
    if constexpr (sizeof(T) == 4) {
        return __uint_as_float(__reduce_max_sync(0xffffffffu, __float_as_uint(v)));
    } else {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const T w = __shfl_xor_sync(0xffffffffu, v, o);
            v = w > v ? w : v;
        }
        return v;
    }
}

template <typename A>
__device__ __forceinline__ A warp_sum(A v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// --------------------------------------------------------------------------
// The step kernel.

template <typename T>
__device__ __forceinline__ T qnan_of();
template <>
__device__ __forceinline__ float qnan_of<float>()
{
    return __int_as_float(0x7fc00000);
}
template <>
__device__ __forceinline__ double qnan_of<double>()
{
    return __longlong_as_double(0x7ff8000000000000ll);
}

// A*x accumulated in the accumulator precision: double products for the
// reference's double accumulators, float products for the all-FP32 variant.
template <typename AccT, typename T>
__device__ __forceinline__ AccT acc_mul(T a, T x)
{
    if constexpr (sizeof(AccT) == 8)
        return (double)a * (double)x;
    else
        return (float)(a * x);
}

// Per-step values every warp of a step reads (from the control block).
template <typename T>
struct StepVals {
    StepK<T> k;
    T dt, A, F, tmax_val, inflow_dh, rainv, dd, qnan;
    T vseed;                     // prune dt candidates below this velocity (0: none)
    int want_v;
    const T *hin;
    T *hout;
};

template <typename T, int K>
__device__ __forceinline__ StepVals<T> step_vals(const GridD<T> &g, const RunK<T> &rk,
                                                const Ctl *ctl, bool use_seed = true)
{
    StepVals<T> v;
    v.k = rk.k;
    v.k.dt = (T)ctl->dt;
    v.k.den = (T)(2 * K) * v.k.dt;
    v.k.rden = T(1) / v.k.den;
    v.dt = v.k.dt;
    v.A = v.k.A;
    v.F = (T)ctl->F;
    v.tmax_val = (T)ctl->tmax_val;
    v.inflow_dh = (T)ctl->inflow_dh;
    v.want_v = ctl->want_v;
    v.hin = ctl->h_cur ? g.h1 : g.h0;
    v.hout = ctl->h_cur ? g.h0 : g.h1;
    v.rainv = rk.cr_uniform * v.F;   // C*Rday*F for a uniform field
    v.dd = v.k.d_diag;
    v.qnan = qnan_of<T>();
    if (use_seed) {
        if constexpr (sizeof(T) == 4)
            v.vseed = (T)__uint_as_float((unsigned)ctl->vseed_bits);
        else
            v.vseed = (T)__longlong_as_double((long long)ctl->vseed_bits);
    } else {
        v.vseed = T(0);
    }
    return v;
}

// The next-step velocity of one flagged cell given its largest level
// differences to orthogonal (mo) and diagonal (md) neighbours: a cheap upper
// bound first, the exact velocity only when it could raise the running
// maximum (FloodCA src/kernels/physics.h:158-217 for the formulas).
template <typename T, int K, int MATH>
__device__ __forceinline__ T dt_cell(T hv, T nv, T mo, T md, const StepK<T> &k, T dd, T vmax,
                                     T vseed)
{
    T Sb = mo * k.rdx;
    if constexpr (K == 8) {
        const T sd = md * k.rdd;
        Sb = sd > Sb ? sd : Sb;
    }
    if (cell_velocity_bound<T>(hv, nv, Sb * T(1.000001), k) <= (vmax > vseed ? vmax : vseed))
        return vmax;
    T Smax = Mth<T, MATH>::div(mo, k.dx);
    if constexpr (K == 8) {
        const T Sd = Mth<T, MATH>::div(md, dd);
        if (Sd > Smax)
            Smax = Sd;
    }
    const T v = cell_velocity<T, MATH>(hv, nv, Smax, k);
    return v > vmax ? v : vmax;
}

template <typename T, int K, int MATH>
__device__ __noinline__ T dt_cell_out(T hv, T nv, T mo, T md, const StepK<T> k, T dd, T vmax,
                                      T vseed)
{
    return dt_cell<T, K, MATH>(hv, nv, mo, md, k, dd, vmax, vseed);
}

// A warp's running sums over the cells it writes.
template <typename T, typename AccT>
struct StepSums {
    AccT a_rain = 0, a_clamp = 0, a_sea = 0, a_bnd = 0;
    double rain_sum = 0.0;       // sum of rain depths (per-cell rain field)
    long long rain_cells = 0;    // LAND output cells (uniform rain)
    unsigned capn = 0;
    T vmax = T(0);
};

// One warp streams output rows [r0, r1) of one strip through the pipeline.
// LANDONLY: every cell of the grid is LAND; the mask is not read and the
// padding around the grid carries z = PAD_Z (> any terrain), h = 0, which
// makes every face to it carry zero discharge (hf = max(L) - max(z) = 0).
template <typename T, typename AccT, int K, int CPL, int MATH, bool RAINF, bool LANDONLY>
__device__ __forceinline__ void sweep_segment(const GridD<T> &g, const RunK<T> &rk,
                                              const StepVals<T> &sv, int strip, int r0, int r1,
                                              int lane, StepSums<T, AccT> &ss)
{
    using G = Geom<CPL>;
    const StepK<T> &k = sv.k;
    const T dt = sv.dt, A = sv.A, F = sv.F, tmax_val = sv.tmax_val, inflow_dh = sv.inflow_dh;
    const T rainv = sv.rainv, dd = sv.dd, qnan = sv.qnan, vseed = sv.vseed;
    const int want_v = sv.want_v;
    const T *hin = sv.hin;
    T *hout = sv.hout;
    const int nr = g.nr, nc = g.nc;
    AccT &a_clamp = ss.a_clamp, &a_sea = ss.a_sea, &a_bnd = ss.a_bnd, &a_rain = ss.a_rain;
    double &rain_sum = ss.rain_sum;
    long long &rain_cells = ss.rain_cells;
    unsigned &capn = ss.capn;
    T &vmax = ss.vmax;
    (void)a_rain;
    (void)rain_sum;

    const int cbase = strip * G::OW - G::HL + lane * CPL;   // first column of the lane
    const bool out_lane = lane * CPL >= G::HL && lane * CPL < G::HL + G::OW;
    const long long colo = (long long)(cbase + PADC);
    // columns of this lane inside the grid (padding columns are WALL in the
    // generic layout, but LAND-like in the LANDONLY layout)
    bool colok[CPL];
#pragma unroll
    for (int j = 0; j < CPL; j++)
        colok[j] = !LANDONLY || (cbase + j >= 0 && cbase + j < nc);
    // does this lane hold column 0 or column nc-1 (open-edge candidates)?
    const bool edge_lane = (cbase <= 0 && cbase + CPL > 0) || (cbase <= nc - 1 && cbase + CPL > nc - 1);

    // Pipeline registers; the comments give the rows they hold while
    // iteration i runs stages C..E (face rows are the upper cell's row).
    Row<T, CPL> nx, cu, p1, p2, p3;      // rows i+1, i, i-1, i-2, i-3
    T X1[CPL], X2[CPL];                  // x-faces of rows i-1, i-2
    T Y1[CPL], Y2[CPL];                  // y-faces of rows i-2, i-3
    T E1[CPL], E2[CPL];                  // K=8 SE faces of rows i-2, i-3
    T W1[CPL], W2[CPL];                  // K=8 SW faces of rows i-2, i-3
    T s1[CPL], s2[CPL];                  // limiter of rows i-2, i-3
    T qo1[CPL];                          // open-edge discharge of row i-2
    int ko1[CPL];                        // open sides of row i-2
    T L3[CPL], L4[CPL];                  // new level (NaN: WALL) of rows i-3, i-4
    T hn3[CPL];                          // new depth of row i-3
    unsigned eflag = 0u;                 // stage-E candidates of row i-3 (bit per column)
    T hm[CPL];                           // hmax of row i-2
    T cr1[CPL];                          // rain field of row i-2
#pragma unroll
    for (int j = 0; j < CPL; j++) {
        X1[j] = X2[j] = Y1[j] = Y2[j] = T(0);
        E1[j] = E2[j] = W1[j] = W2[j] = T(0);
        s1[j] = s2[j] = T(1);
        qo1[j] = T(0);
        ko1[j] = 0;
        L3[j] = L4[j] = qnan;
        hn3[j] = T(0);
        hm[j] = T(0);
        cr1[j] = T(0);
        cu.z[j] = cu.h[j] = cu.n[j] = T(0);
        cu.m[j] = M_WALL;
    }
    p1 = cu;
    p2 = cu;
    p3 = cu;
    load_row<T, CPL, LANDONLY>(nx, g, hin, (long long)(r0 - 3 + PADR) * g.pitch + colo);

    for (int i = r0 - 3; i <= r1 + 2; i++) {
        p3 = p2;
        p2 = p1;
        p1 = cu;
        cu = nx;
        load_row<T, CPL, LANDONLY>(nx, g, hin, (long long)(i + 1 + PADR) * g.pitch + colo);
        {
            // L2 prefetch of the row loaded three iterations from now, so
            // that load waits for L2 rather than HBM (no registers held).
            // Measured at 4096^2 on a B200: +2 % exact, +10 % fast math;
            // 3 rows ahead beat 4, 6 and 8. Clamped to the last padding row.
            const int ra = min(i + 1 + PF_ROWS, nr + PADR - 1);
            const long long offa = (long long)(ra + PADR) * g.pitch + colo;
            prefetch_l2(g.z + offa);
            prefetch_l2(hin + offa);
            prefetch_l2(g.n + offa);
        }
        const bool row0_out = i >= r0 && i < r1;
        const bool row1_out = i - 1 >= r0 && i - 1 < r1;
        const bool row2_out = i - 2 >= r0 && i - 2 < r1;
        // hmax and rain field of row i-1, used by stage D next iteration
        const long long off1 = (long long)(i - 1 + PADR) * g.pitch + colo;
        T hm_next[CPL], cr_next[CPL];
        if (row1_out && out_lane)
            VecIO<T, CPL>::ld_rw(hm_next, g.hmax + off1);
        if constexpr (RAINF)
            VecIO<T, CPL>::ld(cr_next, g.cr + off1);

        // ---- A: x-faces of row i; y and diagonal faces of row i-1,
        //      all evaluated together (faces_q) for instruction-level
        //      parallelism across the NF independent faces
        T X0[CPL], Yn[CPL], En[CPL], Wn[CPL];
        {
            constexpr int NF = (K == 8 ? 4 : 2) * CPL;
            const T cz = sh_dn(cu.z[0]), ch = sh_dn(cu.h[0]), cn = sh_dn(cu.n[0]);
            const uint32_t cm = LANDONLY ? (uint32_t)M_LAND : sh_dn(cu.m[0]);
            T pz = T(0), ph = T(0), pn = T(0);
            uint32_t pm = M_LAND;
            if constexpr (K == 8) {
                pz = sh_dn(p1.z[0]);
                ph = sh_dn(p1.h[0]);
                pn = sh_dn(p1.n[0]);
                if constexpr (!LANDONLY)
                    pm = sh_dn(p1.m[0]);
            }
            T fza[NF], fha[NF], fna[NF], fzb[NF], fhb[NF], fnb[NF], fd[NF], frd[NF];
            uint32_t fma_[NF], fmb[NF];
#pragma unroll
            for (int j = 0; j < CPL; j++) {
                const T zr = right_of<T, CPL>(cu.z, j, cz), hr = right_of<T, CPL>(cu.h, j, ch);
                const T nrr = right_of<T, CPL>(cu.n, j, cn);
                const uint32_t mr = right_of<uint32_t, CPL>(cu.m, j, cm);
                // x-face (i, c) -> (i, c+1)
                fza[j] = cu.z[j]; fha[j] = cu.h[j]; fna[j] = cu.n[j]; fma_[j] = cu.m[j];
                fzb[j] = zr; fhb[j] = hr; fnb[j] = nrr; fmb[j] = mr;
                fd[j] = k.dx; frd[j] = k.rdx;
                // y-face (i-1, c) -> (i, c)
                const int y = CPL + j;
                fza[y] = p1.z[j]; fha[y] = p1.h[j]; fna[y] = p1.n[j]; fma_[y] = p1.m[j];
                fzb[y] = cu.z[j]; fhb[y] = cu.h[j]; fnb[y] = cu.n[j]; fmb[y] = cu.m[j];
                fd[y] = k.dx; frd[y] = k.rdx;
                if constexpr (K == 8) {
                    // SE face (i-1, c) -> (i, c+1)
                    const int e = 2 * CPL + j;
                    fza[e] = p1.z[j]; fha[e] = p1.h[j]; fna[e] = p1.n[j]; fma_[e] = p1.m[j];
                    fzb[e] = zr; fhb[e] = hr; fnb[e] = nrr; fmb[e] = mr;
                    fd[e] = dd; frd[e] = k.rdd;
                    // SW face (i-1, c+1) -> (i, c)
                    const int w = 3 * CPL + j;
                    fza[w] = right_of<T, CPL>(p1.z, j, pz);
                    fha[w] = right_of<T, CPL>(p1.h, j, ph);
                    fna[w] = right_of<T, CPL>(p1.n, j, pn);
                    fma_[w] = right_of<uint32_t, CPL>(p1.m, j, pm);
                    fzb[w] = cu.z[j]; fhb[w] = cu.h[j]; fnb[w] = cu.n[j]; fmb[w] = cu.m[j];
                    fd[w] = dd; frd[w] = k.rdd;
                }
            }
            T fq[NF];
            unsigned fc[NF];
            faces_q<T, MATH, LANDONLY, NF>(fza, fha, fna, fma_, fzb, fhb, fnb, fmb, fd, frd, k,
                                           fq, fc);
            unsigned c0 = 0u, c1 = 0u;
#pragma unroll
            for (int j = 0; j < CPL; j++) {
                X0[j] = fq[j];
                Yn[j] = fq[CPL + j];
                c0 += fc[j];
                c1 += fc[CPL + j];
                if constexpr (K == 8) {
                    En[j] = fq[2 * CPL + j];
                    Wn[j] = fq[3 * CPL + j];
                    c1 += fc[2 * CPL + j] + fc[3 * CPL + j];
                } else {
                    En[j] = Wn[j] = T(0);
                }
            }
            if (out_lane) {
                if (row0_out)
                    capn += c0;
                if (row1_out)
                    capn += c1;
            }
        }

        // ---- C: outflow and limiter of row i-1, in the reference face
        //      order +x, -x, +y, -y, [d1+, d1-, d2+, d2-], open slots
        T s0[CPL], qo0[CPL];
        int ko0[CPL];
        {
            const T xl = sh_up(X1[CPL - 1]);
            T el = T(0), wl = T(0);
            if constexpr (K == 8) {
                el = sh_up(E1[CPL - 1]);
                wl = sh_up(Wn[CPL - 1]);
            }
            const int r = i - 1;
            const bool edge_row = rk.open && ((r == 0 && rk.edge_n) || (r == nr - 1 && rk.edge_s));
#pragma unroll
            for (int j = 0; j < CPL; j++) {
                const int c = cbase + j;
                int kop = 0;
                if ((edge_row || edge_lane) && rk.open && p1.m[j] == M_LAND)
                    kop = (c == 0 && rk.edge_w) + (c == nc - 1 && rk.edge_e) +
                          (r == 0 && rk.edge_n) + (r == nr - 1 && rk.edge_s);
                T qo = T(0);
                if (kop) {
                    int cap;
                    qo = open_q<T, MATH>(p1.z[j], p1.h[j], p1.n[j], p1.m[j], k, cap);
                    if (row1_out && out_lane)
                        capn += (unsigned)(cap * kop);
                }
                qo0[j] = qo;
                ko0[j] = kop;
                // positive outgoing parts in the reference order; adding a
                // zero leaves a non-negative sum unchanged
                T out = T(0);
                out += fmax(X1[j], T(0));
                out += fmax(-left_of<T, CPL>(X1, j, xl), T(0));
                out += fmax(Yn[j], T(0));
                out += fmax(-Y1[j], T(0));
                if constexpr (K == 8) {
                    out += fmax(En[j], T(0));
                    out += fmax(-left_of<T, CPL>(E1, j, el), T(0));
                    out += fmax(left_of<T, CPL>(Wn, j, wl), T(0));
                    out += fmax(-W1[j], T(0));
                }
                out += open_sum<T>(qo, kop);
                const T ov = out * dt;
                s0[j] = p1.m[j] == M_LAND ? limiter_bf<T, MATH>(ov, p1.h[j], A) : T(1);
            }
        }

        unsigned eflag_next = 0u;
        // ---- D: limiter-scaled net inflow and depth update of row i-2
        //      (s0: row i-1 below, s1: the row itself, s2: row i-3 above)
        T hn2[CPL], Ln2[CPL];
        {
            const int r = i - 2;
            const T sl = sh_up(s1[CPL - 1]), sr = sh_dn(s1[0]);
            const T xl = sh_up(X2[CPL - 1]);
            T bl = T(1), br = T(1), al = T(1), ar = T(1), el = T(0), wl = T(0);
            if constexpr (K == 8) {
                bl = sh_up(s0[CPL - 1]);
                br = sh_dn(s0[0]);
                al = sh_up(s2[CPL - 1]);
                ar = sh_dn(s2[0]);
                el = sh_up(E2[CPL - 1]);
                wl = sh_up(W1[CPL - 1]);
            }
            uint32_t ml = 0, mr = 0, m1l = 0, m1r = 0, m3l = 0, m3r = 0;
            if (rk.has_sea) {
                ml = sh_up(p2.m[CPL - 1]);
                mr = sh_dn(p2.m[0]);
                if constexpr (K == 8) {
                    m1l = sh_up(p1.m[CPL - 1]);
                    m1r = sh_dn(p1.m[0]);
                    m3l = sh_up(p3.m[CPL - 1]);
                    m3r = sh_dn(p3.m[0]);
                }
            }
            const bool sea_on = rk.has_sea != 0;
            const bool inflow_row = r == rk.inflow_r;
            // open-edge terms exist only on open edge rows or edge lanes
            const bool open2 = edge_lane || (rk.open && ((r == 0 && rk.edge_n) ||
                                                         (r == nr - 1 && rk.edge_s)));
            const bool row2_in = r >= g.r_lo && r < g.r_hi;
            // stage-E threshold: the warp's running velocity maximum
            T thr = want_v ? warp_max_nonneg(vmax) : T(0);
            thr = thr > vseed ? thr : vseed;
            T *tm_row = g.tmax + (long long)(r + PADR) * g.pitch + colo;
            bool rose_any = false, bnd_open = false;
            T qbnd[CPL];
            if constexpr (LANDONLY && sizeof(AccT) == 8 && !RAINF) {
                if (row2_out && out_lane) {
#pragma unroll
                    for (int j = 0; j < CPL; j++)
                        rain_cells += colok[j] ? 1 : 0;
                }
            }
            T hmx[CPL];
#pragma unroll
            for (int j = 0; j < CPL; j++) {
                const uint32_t ma = p2.m[j];
                const bool land = ma == M_LAND;
                const T sa = s1[j];
                T net = T(0), Q, Qs;
                double sea = 0.0;
                // +x: face (r, c) -> (r, c+1)
                Q = X2[j];
                Qs = Q * (Q >= T(0) ? sa : right_of<T, CPL>(s1, j, sr));
                net -= Qs;
                if (sea_on && land && right_of<uint32_t, CPL>(p2.m, j, mr) == M_SEA && Qs > T(0))
                    sea += (double)dt * (double)Qs;
                // -x: face (r, c-1) -> (r, c)
                Q = left_of<T, CPL>(X2, j, xl);
                Qs = Q * (Q >= T(0) ? left_of<T, CPL>(s1, j, sl) : sa);
                net += Qs;
                if (sea_on && land && left_of<uint32_t, CPL>(p2.m, j, ml) == M_SEA && Qs < T(0))
                    sea += (double)dt * (double)(-Qs);
                // +y: face (r, c) -> (r+1, c)
                Q = Y1[j];
                Qs = Q * (Q >= T(0) ? sa : s0[j]);
                net -= Qs;
                if (sea_on && land && p1.m[j] == M_SEA && Qs > T(0))
                    sea += (double)dt * (double)Qs;
                // -y: face (r-1, c) -> (r, c)
                Q = Y2[j];
                Qs = Q * (Q >= T(0) ? s2[j] : sa);
                net += Qs;
                if (sea_on && land && p3.m[j] == M_SEA && Qs < T(0))
                    sea += (double)dt * (double)(-Qs);
                if constexpr (K == 8) {
                    // d1+: (r, c) -> (r+1, c+1)
                    Q = E1[j];
                    Qs = Q * (Q >= T(0) ? sa : right_of<T, CPL>(s0, j, br));
                    net -= Qs;
                    if (sea_on && land && right_of<uint32_t, CPL>(p1.m, j, m1r) == M_SEA &&
                        Qs > T(0))
                        sea += (double)dt * (double)Qs;
                    // d1-: (r-1, c-1) -> (r, c)
                    Q = left_of<T, CPL>(E2, j, el);
                    Qs = Q * (Q >= T(0) ? left_of<T, CPL>(s2, j, al) : sa);
                    net += Qs;
                    if (sea_on && land && left_of<uint32_t, CPL>(p3.m, j, m3l) == M_SEA &&
                        Qs < T(0))
                        sea += (double)dt * (double)(-Qs);
                    // d2+: (r, c) -> (r+1, c-1), SW face of index (r, c-1)
                    Q = left_of<T, CPL>(W1, j, wl);
                    Qs = Q * (Q >= T(0) ? sa : left_of<T, CPL>(s0, j, bl));
                    net -= Qs;
                    if (sea_on && land && left_of<uint32_t, CPL>(p1.m, j, m1l) == M_SEA &&
                        Qs > T(0))
                        sea += (double)dt * (double)Qs;
                    // d2-: (r-1, c+1) -> (r, c), SW face of index (r-1, c)
                    Q = W2[j];
                    Qs = Q * (Q >= T(0) ? right_of<T, CPL>(s2, j, ar) : sa);
                    net += Qs;
                    if (sea_on && land && right_of<uint32_t, CPL>(p3.m, j, m3r) == M_SEA &&
                        Qs < T(0))
                        sea += (double)dt * (double)(-Qs);
                }
                T Qo = T(0);
                if (open2) {
                    Qo = open_sum<T>(qo1[j] * sa, ko1[j]);
                    net -= Qo;
                }
                const bool cell_out = row2_out && out_lane && colok[j];
                T ha = p2.h[j];
                const T rain = RAINF ? cr1[j] * F : rainv;
                T hu = ha + (dt * Mth<T, MATH>::div_c(net, A, k.inv_A) + rain);
                hu = land ? hu : ha;
                // rare events are settled after the loop: clamp, open edge, sea
                if (land && hu < T(0)) {
                    if (cell_out)
                        a_clamp += acc_mul<AccT, T>(-hu, A);
                    hu = T(0);
                }
                ha = hu;
                if (inflow_row && land && cbase + j == rk.inflow_c)
                    ha = ha + inflow_dh;
                if constexpr (sizeof(AccT) == 4) {
                    if (cell_out && land)
                        a_rain += A * rain;
                } else if constexpr (RAINF) {
                    rain_sum += (cell_out && land) ? (double)rain : 0.0;
                } else if constexpr (!LANDONLY) {
                    rain_cells += (cell_out && land) ? 1 : 0;
                }
                if (sea_on && cell_out)
                    a_sea += (AccT)sea;
                if (open2)
                    bnd_open |= cell_out && ko1[j] != 0;
                qbnd[j] = Qo;
                if constexpr (LANDONLY) {
                    // outside the grid: keep the padding depth, no face
                    const bool inside = colok[j] && row2_in;
                    hn2[j] = inside ? ha : p2.h[j];
                    Ln2[j] = inside ? p2.z[j] + ha : qnan;
                } else {
                    hn2[j] = ha;
                    Ln2[j] = ma == M_WALL ? qnan : (ma == M_SEA ? k.z_sea : p2.z[j] + ha);
                }
                // prefilter of the next dt: a cell whose critical velocity
                // sqrt(g h) is surely below thr cannot raise the maximum
                // (g h <= thr^2 (1 - 1e-6): the margin covers the rounding of
                // both products and of the square root by far); flagged
                // cells get the exact evaluation in stage E
                if (want_v && cell_out && land && ha >= k.tau_h &&
                    !(thr > T(0) && k.g * ha <= thr * thr * T(0.999999)))
                    eflag_next |= 1u << j;
                const bool rise = cell_out && land && ha > hm[j];
                hmx[j] = rise ? ha : hm[j];
                rose_any |= rise;
                if (rise)
                    tm_row[j] = tmax_val;
            }
            if (bnd_open) {
#pragma unroll
                for (int j = 0; j < CPL; j++)
                    if (row2_out && out_lane && colok[j] && ko1[j])
                        a_bnd += acc_mul<AccT, T>(dt, qbnd[j]);
            }
            if (row2_out && out_lane) {
                const long long off2 = (long long)(r + PADR) * g.pitch + colo;
                VecIO<T, CPL>::st(hout + off2, hn2);
                if (rose_any)
                    VecIO<T, CPL>::st(g.hmax + off2, hmx);
            }
        }

        // ---- E: next step's stable velocity of row i-3 from the new
        //      levels of rows i-4 (L4), i-3 (L3) and i-2 (Ln2), for the
        //      cells stage D flagged: wet LAND output cells whose critical
        //      velocity could exceed the warp's running maximum (every
        //      other cell's velocity is capped below it).
        if (want_v && __any_sync(0xffffffffu, eflag != 0u)) {
            const int r = i - 3;
            vmax = warp_max_nonneg(vmax);
            const T Ll = sh_up(L3[CPL - 1]), Lr = sh_dn(L3[0]);
            T L2l = T(0), L2r = T(0), L4l = T(0), L4r = T(0);
            if constexpr (K == 8) {
                L2l = sh_up(Ln2[CPL - 1]);
                L2r = sh_dn(Ln2[0]);
                L4l = sh_up(L4[CPL - 1]);
                L4r = sh_dn(L4[0]);
            }
            const bool edge_row = rk.open && ((r == 0 && rk.edge_n) || (r == nr - 1 && rk.edge_s));
#pragma unroll
            for (int j = 0; j < CPL; j++) {
                if (!(eflag & (1u << j)))
                    continue;
                const T hv = hn3[j];
                const int c = cbase + j;
                const T la = L3[j];
                T mo = T(0);
                mo = fmax(mo, fabs(la - right_of<T, CPL>(L3, j, Lr)));
                mo = fmax(mo, fabs(la - left_of<T, CPL>(L3, j, Ll)));
                mo = fmax(mo, fabs(la - Ln2[j]));
                mo = fmax(mo, fabs(la - L4[j]));
                if (edge_row || (edge_lane && rk.open &&
                                 ((c == 0 && rk.edge_w) || (c == nc - 1 && rk.edge_e)))) {
                    const T lv = p3.z[j] - k.S_bnd * k.dx;
                    mo = fmax(mo, fabs(la - lv));
                }
                T md = T(0);
                if constexpr (K == 8) {
                    md = fmax(md, fabs(la - right_of<T, CPL>(Ln2, j, L2r)));
                    md = fmax(md, fabs(la - left_of<T, CPL>(Ln2, j, L2l)));
                    md = fmax(md, fabs(la - right_of<T, CPL>(L4, j, L4r)));
                    md = fmax(md, fabs(la - left_of<T, CPL>(L4, j, L4l)));
                }
                // K = 8 evaluates the cell out of line: fewer live registers
                // in the sweep (measured 3 % faster for K = 8 at 4096^2 on a
                // B200, 6 % slower for K = 4)
                if constexpr (K == 8)
                    vmax = dt_cell_out<T, K, MATH>(hv, p3.n[j], mo, md, k, dd, vmax, vseed);
                else
                    vmax = dt_cell<T, K, MATH>(hv, p3.n[j], mo, md, k, dd, vmax, vseed);
            }
        }

        // ---- advance the pipeline
#pragma unroll
        for (int j = 0; j < CPL; j++) {
            X2[j] = X1[j];
            X1[j] = X0[j];
            Y2[j] = Y1[j];
            Y1[j] = Yn[j];
            if constexpr (K == 8) {
                E2[j] = E1[j];
                E1[j] = En[j];
                W2[j] = W1[j];
                W1[j] = Wn[j];
            }
            s2[j] = s1[j];
            s1[j] = s0[j];
            qo1[j] = qo0[j];
            ko1[j] = ko0[j];
            L4[j] = L3[j];
            L3[j] = Ln2[j];
            hn3[j] = hn2[j];
            eflag = eflag_next;
            if (row1_out && out_lane)
                hm[j] = hm_next[j];
            if constexpr (RAINF)
                cr1[j] = cr_next[j];
        }
    }
}

// Publishes a warp's sums to a control block: accumulator slot `slot`,
// velocity maximum for the next dt.
template <typename T, typename AccT, bool RAINF>
__device__ __forceinline__ void publish_sums(StepSums<T, AccT> &ss, const StepVals<T> &sv,
                                             Ctl *ctl, int lane, int slot)
{
    AccT a_rain = ss.a_rain;
    if constexpr (sizeof(AccT) == 8) {
        if constexpr (RAINF)
            a_rain = (double)sv.A * ss.rain_sum;
        else
            a_rain = (double)ss.rain_cells * ((double)sv.A * (double)sv.rainv);
    }
    a_rain = warp_sum(a_rain);
    const AccT a_clamp = warp_sum(ss.a_clamp);
    const AccT a_sea = warp_sum(ss.a_sea);
    const AccT a_bnd = warp_sum(ss.a_bnd);
    const unsigned capn = warp_sum(ss.capn);
    T vmax = ss.vmax;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const T vo = __shfl_xor_sync(0xffffffffu, vmax, o);
        vmax = vo > vmax ? vo : vmax;
    }
    if (lane == 0) {
        if constexpr (sizeof(AccT) == 8) {
            if (a_rain != 0) atomicAdd(&ctl->accd[0][slot], (double)a_rain);
            if (a_clamp != 0) atomicAdd(&ctl->accd[1][slot], (double)a_clamp);
            if (a_sea != 0) atomicAdd(&ctl->accd[2][slot], (double)a_sea);
            if (a_bnd != 0) atomicAdd(&ctl->accd[3][slot], (double)a_bnd);
        } else {
            if (a_rain != 0) atomicAdd(&ctl->accf[0][slot], (float)a_rain);
            if (a_clamp != 0) atomicAdd(&ctl->accf[1][slot], (float)a_clamp);
            if (a_sea != 0) atomicAdd(&ctl->accf[2][slot], (float)a_sea);
            if (a_bnd != 0) atomicAdd(&ctl->accf[3][slot], (float)a_bnd);
        }
        if (capn)
            atomicAdd(&ctl->cap[slot], (unsigned long long)capn);
        if (sv.want_v && vmax > T(0)) {
            if constexpr (sizeof(T) == 4)
                atomicMax(&ctl->vmax_bits, (unsigned long long)__float_as_uint((float)vmax));
            else
                atomicMax(&ctl->vmax_bits, (unsigned long long)__double_as_longlong((double)vmax));
        }
    }
}

}  // namespace fcab

#include "wca_sweep_f2.cuh"
#include "wca_sweep_f4.cuh"

namespace fcab {

// The pair sweep runs the FP32 all-LAND K = 4 grids at two columns per
// lane; every other variant runs sweep_segment (all of them with
// FCAB_PAIR_SWEEP=0, a build option for comparing the two).
#ifndef FCAB_PAIR_SWEEP
#define FCAB_PAIR_SWEEP 1
#endif
// For K = 8 the scalar sweep is the faster of the two (measured at 4096^2
// on a B200: 24.8 against 23.4 Gcell/s exact, 36.4 against 32.5 fast; the
// pair sweep's K = 8 face state leaves it 8 warps per SM); FCAB_PAIR_K8=1
// runs K = 8 on the pair sweep too.
#ifndef FCAB_PAIR_K8
#define FCAB_PAIR_K8 0
#endif
template <typename T, int K, int CPL, bool LANDONLY>
__host__ __device__ constexpr bool use_pair_sweep()
{
    return FCAB_PAIR_SWEEP && sizeof(T) == 4 && CPL == 2 && LANDONLY && (K == 4 || FCAB_PAIR_K8);
}
// The four-column sweep (two pairs per lane) runs the FP32 all-LAND K = 4
// grids at four columns per lane.
template <typename T, int K, int CPL, bool LANDONLY>
__host__ __device__ constexpr bool use_quad_sweep()
{
    return FCAB_PAIR_SWEEP && sizeof(T) == 4 && CPL == 4 && K == 4 && LANDONLY;
}

// Launch shape of the step kernel: threads per CTA and the resident warps
// per SM the register allocation aims for (65536 / (32 x warps) registers
// per thread). Measured at 4096^2 on a B200: the exact CPL-2 kernel runs 15 %
// faster with 16 warps (128 registers, 32 B of spills) than with 12; the fast
// one 3 % slower.
#ifndef FCAB_STEP_THREADS
#define FCAB_STEP_THREADS 128
#endif
#ifndef FCAB_STEP_WARPS
#define FCAB_STEP_WARPS 0
#endif
template <int CPL, int MATH>
__host__ __device__ constexpr int step_threads()
{
    return FCAB_STEP_THREADS;
}
template <int K, int CPL, int MATH>
__host__ __device__ constexpr int step_min_blocks()
{
    // K = 8 exact at CPL 2 spills 56 B at 16 warps and runs 3.5 % faster at 12
    return (FCAB_STEP_WARPS > 0
                ? FCAB_STEP_WARPS
                : (CPL == 1 ? 16
                            : CPL == 2 ? (MATH == MATH_EXACT && K == 4 ? 16 : 12) : 8)) /
           (step_threads<CPL, MATH>() / 32);
}
// Resident warps per SM the pair sweep's register allocation aims for.
// Measured at 4096^2 on a B200 (one-row loop, same box): 16 warps (128
// registers, about 160 B of spill stores) 44.4-45.1 Gcell/s, 12 warps (160
// registers, no spills) 41.2-41.4, 20 warps (96 registers, 532 B of
// spills) 37.4, 8 warps 30.5-31.3: occupancy outweighs the spills up to 16.
#ifndef FCAB_PAIR_WARPS
#define FCAB_PAIR_WARPS 16
#endif
// K = 8 holds twice the face state: 8 warps (up to 255 registers, no spills)
#ifndef FCAB_PAIR_WARPS_K8
#define FCAB_PAIR_WARPS_K8 8
#endif
template <int K>
__host__ __device__ constexpr int pair_warps()
{
    return K == 8 ? FCAB_PAIR_WARPS_K8 : FCAB_PAIR_WARPS;
}
// The batched step keeps a member descriptor and step constants per warp
// besides the sweep state. With stage E's depth and n and the hmax row out
// of the register ring it spills 108 B at 16 warps (128 registers), and the
// config-4 ensemble (256 members) ran 50.9 G cell-steps/s against 48.8 at
// 12 warps (168 registers, no spills) on one box.
#ifndef FCAB_PAIR_WARPS_BATCH
#define FCAB_PAIR_WARPS_BATCH 16
#endif
template <int K>
__host__ __device__ constexpr int pair_warps_batch()
{
    return K == 8 ? FCAB_PAIR_WARPS_K8 : FCAB_PAIR_WARPS_BATCH;
}
// Resident warps per SM of the four-column sweep (twice the pair sweep's
// state per lane: up to 255 registers at 8 warps)
#ifndef FCAB_QUAD_WARPS
#define FCAB_QUAD_WARPS 8
#endif
template <typename T, int K, int CPL, int MATH, bool LANDONLY>
__host__ __device__ constexpr int step_blocks_per_sm()
{
    return use_pair_sweep<T, K, CPL, LANDONLY>()
               ? pair_warps<K>() / (step_threads<CPL, MATH>() / 32)
               : use_quad_sweep<T, K, CPL, LANDONLY>()
                     ? FCAB_QUAD_WARPS / (step_threads<CPL, MATH>() / 32)
                     : step_min_blocks<K, CPL, MATH>();
}

template <typename T, int K, int MATH>
__global__ void k_init_dt(GridD<T> g, RunK<T> rk, TimeCfg tc, Ctl *ctl, int only_if_needed);

// CTAs of the full velocity pass (grid-stride over every cell; 256 threads)
constexpr int VPASS_GRID = 148 * 8;

template <typename T, typename AccT, int K, int CPL, int MATH, bool RAINF, bool LANDONLY>
__global__ void __launch_bounds__(step_threads<CPL, MATH>(),
                                  step_blocks_per_sm<T, K, CPL, MATH, LANDONLY>()) k_step(GridD<T> g, RunK<T> rk, TimeCfg tc, Ctl *ctl,
                                              int warps_total)
{
    using G = Geom<CPL>;
    if (ctl->active == 0)
        return;
    const int lane = threadIdx.x & 31;
    const int wid = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const StepVals<T> sv = step_vals<T, K>(g, rk, ctl);
    StepSums<T, AccT> ss;

    const int nr = g.nr, nc = g.nc;
    const int nstrips = (nc + G::OW - 1) / G::OW;
    const long long total = (long long)nstrips * nr;
    long long w0 = total * wid / warps_total, w1 = total * (wid + 1) / warps_total;
    if (wid >= warps_total)
        w0 = w1 = 0;

    // step constants in shared memory for the pair sweep's exact
    // re-evaluations; the warps' TMA rings and barriers (dynamic shared memory)
    __shared__ StepK<T> sk;
    __shared__ uint32_t tphase[step_threads<CPL, MATH>() / 32];
    __shared__ int tma_bad;
    extern __shared__ __align__(1024) unsigned char fcab_dsm[];
    uint32_t ring = 0u, bars = 0u;
    const int wib = threadIdx.x >> 5;
    if constexpr (use_quad_sweep<T, K, CPL, LANDONLY>()) {
        if (threadIdx.x == 0)
            sk = sv.k;
        __syncthreads();
    }
    if constexpr (use_pair_sweep<T, K, CPL, LANDONLY>()) {
        if (threadIdx.x == 0) {
            sk = sv.k;
            tma_bad = 0;
        }
        // TMA destinations must start on 128-byte boundaries: the rings
        // start at the dynamic area rounded up to 1024 bytes (the area has
        // 1 KB of slack for it)
        const uint32_t dbase = (smem_addr(fcab_dsm) + 1023u) & ~1023u;
        if (g.tmap) {
            constexpr int W = step_threads<CPL, MATH>() / 32;
            ring = dbase + wib * TMA_WARP_B;
            bars = dbase + W * TMA_WARP_B + wib * TMA_NS * 8;
            if (lane == 0) {
                for (int q = 0; q < TMA_NS; q++)
                    mbar_init1(bars + 8u * q);
                tphase[wib] = 0u;
                fence_proxy_async_smem();
            }
        }
        __syncthreads();
    }
    while (w0 < w1) {
        const int strip = (int)(w0 / nr);
        const int r0 = (int)(w0 % nr);
        const int r1 = (int)min((long long)nr, (long long)r0 + (w1 - w0));
        w0 += r1 - r0;
        if constexpr (use_pair_sweep<T, K, CPL, LANDONLY>()) {
            bool bad = false;
            PairSweep<AccT, K, MATH, RAINF>::run(g, rk, sv, &sk, strip, r0, r1, lane, ss, ring,
                                                 bars, &tphase[wib], &bad);
            if (bad && lane == 0)
                tma_bad = 1;
        } else if constexpr (use_quad_sweep<T, K, CPL, LANDONLY>()) {
            QuadSweep<AccT, MATH, RAINF>::run(g, rk, sv, &sk, strip, r0, r1, lane, ss);
        } else {
            sweep_segment<T, AccT, K, CPL, MATH, RAINF, LANDONLY>(g, rk, sv, strip, r0, r1, lane,
                                                                  ss);
        }
    }
    if constexpr (use_pair_sweep<T, K, CPL, LANDONLY>()) {
        __syncthreads();
        if (threadIdx.x == 0 && tma_bad)
            ctl->err = 3;           // a row tile never arrived; the host reports it
    }

    publish_sums<T, AccT, RAINF>(ss, sv, ctl, lane, wid & (NSLOT - 1));
    // ---- the last CTA to finish prepares the next step
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned prev = atomicAdd(&ctl->ctas_done, 1u);
        if (prev == gridDim.x - 1) {
            __threadfence();
            ctl->h_cur ^= 1;
            ctl->launches += 1;
            if (tc.split) {
                ctl->fin_pending = 1;
                ctl->ctas_done = 0u;
            } else {
                finalize<T>(ctl, tc, rk, true);
                // a missed seed defers this step's dt to the full velocity
                // pass: launched from here into the tail of the stream, so
                // it runs before the next step and only when needed
                if (tc.tail_vpass && ctl->need_v) {
                    k_init_dt<T, K, MATH><<<VPASS_GRID, 256, 0, cudaStreamTailLaunch>>>(g, rk, tc,
                                                                                      ctl, 1);
                    if (cudaGetLastError() != cudaSuccess)
                        ctl->err = 2;   // the host's poll runs the pass instead
                }
            }
        }
    }
}

// --------------------------------------------------------------------------
// Batched step: one launch advances every active member of an ensemble by
// one step. Members keep their own grids, control blocks, dt and time. Warps
// take work units (member, row block, strip) from an atomic queue; a unit of
// an inactive member (finished, or paused at its window end) is skipped. The
// warp that completes a member's last unit prepares that member's next step.
// The last warp to leave resets the queue for the next launch. No warp ever
// waits for another.

template <typename T>
struct MemberD {
    GridD<T> g;
    RunK<T> rk;
    TimeCfg tc;
    Ctl *ctl;
    int unit_off, units, strips, seg;
};

struct BatchQ {
    unsigned int next_unit;
    unsigned int warps_out;
    unsigned int nneed;         // members whose step deferred its dt (seed missed)
    unsigned int vfull_out;     // CTAs done with the full velocity passes
};

template <typename T, typename AccT, int K, int CPL, int MATH, bool RAINF, bool LANDONLY>
__global__ void __launch_bounds__(128, use_pair_sweep<T, K, CPL, LANDONLY>() ? pair_warps_batch<K>() / 4
                                                                      : (CPL == 2 ? 4 : 1))
k_step_batch(const MemberD<T> *members,
                                                    const int *unit_member, int total_units,
                                                    BatchQ *q, int *need_list)
{
    const int lane = threadIdx.x & 31;
    // The unit's member descriptor and step constants live in the warp's
    // shared-memory slot, not in registers: the compiler reloads them where
    // needed instead of holding ~60 warp-uniform values, which lets 4 CTAs
    // (16 warps) fit per SM (measured on a B200, 64 config-4 members: 39.6
    // against 37.1 G cell-steps/s with register copies at 3 CTAs).
    const int wib = threadIdx.x >> 5;
    __shared__ MemberD<T> smd[4];
    __shared__ StepVals<T> ssv[4];
    static_assert(sizeof(MemberD<T>) % 4 == 0 && sizeof(StepVals<T>) % 4 == 0, "word copies");
    for (;;) {
        unsigned u = 0;
        if (lane == 0)
            u = atomicAdd(&q->next_unit, 1u);
        u = __shfl_sync(0xffffffffu, u, 0);
        if (u >= (unsigned)total_units)
            break;
        const int m = unit_member[u];
        __syncwarp();
        {
            const unsigned *src = reinterpret_cast<const unsigned *>(members + m);
            unsigned *dst = reinterpret_cast<unsigned *>(&smd[wib]);
            for (int w = lane; w < (int)(sizeof(MemberD<T>) / 4); w += 32)
                dst[w] = src[w];
        }
        __syncwarp();
        const MemberD<T> &md = smd[wib];
        Ctl *ctl = md.ctl;
        if (ctl->active == 0)
            continue;
        const GridD<T> &g = md.g;
        const RunK<T> &rk = md.rk;
        const int local = (int)u - md.unit_off;
        const int strip = local % md.strips, blk = local / md.strips;
        const int r0 = blk * md.seg, r1 = min(g.nr, r0 + md.seg);
        {
            const StepVals<T> sv0 = step_vals<T, K>(g, rk, ctl);
            if (lane == 0)
                ssv[wib] = sv0;
        }
        __syncwarp();
        const StepVals<T> &sv = ssv[wib];
        StepSums<T, AccT> ss;
        if constexpr (use_pair_sweep<T, K, CPL, LANDONLY>())
            PairSweep<AccT, K, MATH, RAINF>::run(g, rk, sv, &ssv[wib].k, strip, r0, r1, lane, ss);
        else
            sweep_segment<T, AccT, K, CPL, MATH, RAINF, LANDONLY>(g, rk, sv, strip, r0, r1, lane,
                                                                  ss);
        publish_sums<T, AccT, RAINF>(ss, sv, ctl, lane, (int)(u & (NSLOT - 1)));
        if (lane == 0) {
            __threadfence();
            const unsigned prev = atomicAdd(&ctl->ctas_done, 1u);
            if (prev == (unsigned)md.units - 1u) {
                __threadfence();
                ctl->h_cur ^= 1;
                ctl->launches += 1;
                const TimeCfg tc = md.tc;
                finalize<T>(ctl, tc, rk, true);
                if (ctl->need_v)    // seed missed: the full pass after this launch
                    need_list[atomicAdd(&q->nneed, 1u)] = m;
            }
        }
        __syncwarp();
    }
    if (lane == 0) {
        __threadfence();
        const unsigned nw = gridDim.x * (blockDim.x >> 5);
        if (atomicAdd(&q->warps_out, 1u) == nw - 1u) {
            q->next_unit = 0u;
            q->warps_out = 0u;
        }
    }
}

// Opens the next output window of every member that is not finished.
template <typename T>
__global__ void k_batch_window(const MemberD<T> *members, int n, double window)
{
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= n)
        return;
    Ctl *c = members[m].ctl;
    if (c->done)
        return;
    c->window_end += window;
    if (c->pause && c->t < c->window_end - 1e-9) {
        c->pause = 0;
        c->active = 1;
    }
}

// --------------------------------------------------------------------------
// Full velocity pass: max stable velocity over the current depth (one
// thread per cell), then the step control without a time advance. Run once
// for the first step's dt, and (only_if_needed) after a step whose
// seed-pruned velocity maximum fell below the seed, so that step's dt comes
// from every cell.

template <typename T, int K, int MATH>
__device__ void velocity_pass(const GridD<T> &g, const RunK<T> &rk, const TimeCfg &tc, Ctl *ctl)
{
    const StepK<T> k = rk.k;
    const T *h = ctl->h_cur ? g.h1 : g.h0;
    T vmax = T(0);
    const long long N = (long long)g.nr * g.nc;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < N;
         idx += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(idx / g.nc), c = (int)(idx % g.nc);
        const long long a = (long long)(r + PADR) * g.pitch + c + PADC;
        if (g.m[a] != M_LAND || !(h[a] >= k.tau_h))
            continue;
        const T la = g.z[a] + h[a];
        T mo = T(0), md = T(0);
        const long long nb[8] = {a + 1, a - 1, a + g.pitch, a - g.pitch,
                                 a + g.pitch + 1, a + g.pitch - 1, a - g.pitch + 1,
                                 a - g.pitch - 1};
#pragma unroll
        for (int q = 0; q < (K == 8 ? 8 : 4); q++) {
            const uint32_t mb = g.m[nb[q]];
            if (mb == M_WALL)
                continue;
            const T lb = mb == M_SEA ? k.z_sea : g.z[nb[q]] + h[nb[q]];
            const T d = fabs(la - lb);
            if (q < 4)
                mo = fmax(mo, d);
            else
                md = fmax(md, d);
        }
        if (rk.open && ((c == 0 && rk.edge_w) || (c == g.nc - 1 && rk.edge_e) ||
                        (r == 0 && rk.edge_n) || (r == g.nr - 1 && rk.edge_s)))
            mo = fmax(mo, fabs(la - (g.z[a] - k.S_bnd * k.dx)));
        T Smax = Mth<T, MATH>::div(mo, k.dx);
        if (K == 8) {
            const T Sd = Mth<T, MATH>::div(md, k.d_diag);
            if (Sd > Smax)
                Smax = Sd;
        }
        const T v = cell_velocity<T, MATH>(h[a], g.n[a], Smax, k);
        if (v > vmax)
            vmax = v;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        T vo = __shfl_xor_sync(0xffffffffu, vmax, o);
        vmax = vo > vmax ? vo : vmax;
    }
    if ((threadIdx.x & 31) == 0 && vmax > T(0)) {
        if constexpr (sizeof(T) == 4)
            atomicMax(&ctl->vmax_bits, (unsigned long long)__float_as_uint((float)vmax));
        else
            atomicMax(&ctl->vmax_bits, (unsigned long long)__double_as_longlong((double)vmax));
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned prev = atomicAdd(&ctl->ctas_done, 1u);
        if (prev == gridDim.x - 1) {
            __threadfence();
            if (tc.split) {
                ctl->fin_pending = 2;
                ctl->ctas_done = 0u;
            } else {
                finalize<T>(ctl, tc, rk, false);
            }
        }
    }
}

template <typename T, int K, int MATH>
__global__ void k_init_dt(GridD<T> g, RunK<T> rk, TimeCfg tc, Ctl *ctl, int only_if_needed)
{
    // only_if_needed: the full velocity pass after a step whose pruned
    // maximum fell below its seed (ctl->need_v); otherwise nothing to do
    if (only_if_needed && ctl->need_v == 0)
        return;
    velocity_pass<T, K, MATH>(g, rk, tc, ctl);
}

// The full velocity pass of every batch member whose step deferred its dt
// (need_list, filled by the step launch before), one member after another
// over the whole grid; the last CTA out clears the list.
template <typename T, int K, int MATH>
__global__ void k_batch_vfull(const MemberD<T> *members, const int *need_list, BatchQ *q)
{
    const unsigned nneed = q->nneed;
    for (unsigned i = 0; i < nneed; i++) {
        const MemberD<T> &md = members[need_list[i]];
        velocity_pass<T, K, MATH>(md.g, md.rk, md.tc, md.ctl);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&q->vfull_out, 1u) == gridDim.x - 1u) {
            q->nneed = 0u;
            q->vfull_out = 0u;
        }
    }
}

// LAND volume sum(h*A) in double (FloodCA src/common/grid.c:125-141).
template <typename T>
__global__ void k_volume(GridD<T> g, const Ctl *ctl, T A, double *out)
{
    const T *h = ctl->h_cur ? g.h1 : g.h0;
    double v = 0.0;
    const long long N = (long long)g.nr * g.nc;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < N;
         idx += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(idx / g.nc), c = (int)(idx % g.nc);
        const long long a = (long long)(r + PADR) * g.pitch + c + PADC;
        if (g.m[a] == M_LAND)
            v += (double)h[a] * (double)A;
    }
    v = warp_sum(v);
    if ((threadIdx.x & 31) == 0 && v != 0.0)
        atomicAdd(out, v);
}

// --------------------------------------------------------------------------
// Slabs of a row-split domain. Each slab holds its own rows plus up to three
// halo rows of each neighbour in its padding rows; the step kernel and the
// velocity pass leave the step control pending (fin_pending) with the
// slab's own velocity maximum in vmax_bits. Once vmax_bits holds the maximum
// over all slabs, every slab prepares the same next step here, as one
// domain would (FloodCA src/common/model.c:111-156 reduces dt the same way
// through comm->min_real).

template <typename T>
__global__ void k_slab_finalize(RunK<T> rk, TimeCfg tc, Ctl *ctl)
{
    const int p = ctl->fin_pending;
    if (p == 0)
        return;
    ctl->fin_pending = 0;
    finalize<T>(ctl, tc, rk, p == 1);
}

// Copies rows [row0, row0 + nrows) of the current depth to a dense
// nrows x nc buffer (to_buf) or back; rows may lie in the halo.
template <typename T>
__global__ void k_rows_copy(const Ctl *ctl, T *h0, T *h1, long long pitch, int row0, int nrows,
                            int nc, T *buf, int to_buf)
{
    T *h = ctl->h_cur ? h1 : h0;
    const long long N = (long long)nrows * nc;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N;
         i += (long long)gridDim.x * blockDim.x) {
        const long long a = (long long)(row0 + i / nc + PADR) * pitch + i % nc + PADC;
        if (to_buf)
            buf[i] = h[a];
        else
            h[a] = buf[i];
    }
}

}  // namespace fcab
