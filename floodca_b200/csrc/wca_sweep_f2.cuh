// The FP32 sweep on column pairs for all-LAND grids.
//
// Same work decomposition and the same arithmetic as sweep_segment (one warp
// streams a strip of 64 columns down a range of rows; iteration i loads row
// i+1 and runs A faces of rows i-1/i, C limiter of row i-1, D update of row
// i-2, E next-step velocity of row i-3; FloodCA src/kernels/physics.h and
// src/common/model.c:321-605), organised for instruction count:
//
//  * a lane's two columns are one packed f32x2 register pair, so every add,
//    multiply and fused multiply-add runs on both columns in one instruction
//    (the same rounding per half as the scalar instruction);
//  * the pipeline's rows live in a four-slot register ring (row r in slot
//    (r - i0) & 3 of a four-row pass, turned by two slots after a two-row
//    pass, or rotated one slot per row);
//  * the exact formulas run on pairs with correctly rounded divisions, roots
//    and caps (the volume cap by a Markstein division, the critical velocity
//    from the exact product g*hf when a warp has a face near it); a cube root
//    or critical velocity within 2^-11 ulp of a rounding midpoint flags its
//    half, and a warp with a flagged half re-evaluates those halves with the
//    exact scalar formula (face_q). The limiter divides only where the
//    outflow exceeds the held volume, and the next-step velocity first tests
//    a multiply-only bound h^4 S^3 >= thr^6 n^6;
//  * the upwind-scaled discharge of every face is formed once, as
//    Q- * s_down + Q+ * s_up with Q+ = max(Q, 0), Q- = min(Q, 0) (one of the
//    two products is zero, so this is the reference's Q * s_upwind), and
//    used by both cells of the face;
//  * grid edges, open boundaries, the inflow cell and rows outside the grid
//    are handled in warp-uniform branches that only edge strips and edge
//    rows take.
#pragma once

#include "wca_f2.cuh"
#include "wca_tma.cuh"

namespace fcab {

// TMA row source of the pair sweep: each warp streams its strip's z, h and
// n rows through a ring of TMA_NS stages of TMA_RB rows (64 floats each),
// filled by 2-D tensor loads and drained by shared-memory loads.
constexpr int TMA_RB = 8, TMA_NS = 3;

// Iterations per pass of the pair sweep's loop: 4 unrolls the body over the
// four ring slots (no register copies, four copies of the code); 2 runs two
// bodies and turns the ring by two slots after them; 1 runs one body and
// rotates the ring's registers after each row. Measured at 4096^2 on a
// B200: the one-row loop is faster than four (33.9 against 18.9 Gcell/s at
// 12 warps per SM): the four-row body misses the instruction cache.
#ifndef FCAB_PAIR_UNROLL
#define FCAB_PAIR_UNROLL 1
#endif
constexpr uint32_t TMA_FIELD_B = TMA_RB * 256, TMA_STAGE_B = 3 * TMA_FIELD_B;
constexpr uint32_t TMA_WARP_B = TMA_NS * TMA_STAGE_B;
// dynamic shared memory of a CTA of `warps` warps: 1 KB of slack to round
// the start up to a 1024-byte boundary (the dynamic area follows the static
// shared variables, so its own start is only 16-byte aligned), the rings,
// then the barriers
__host__ __device__ constexpr int tma_smem_bytes(int warps)
{
    return 1024 + warps * (int)TMA_WARP_B + warps * TMA_NS * 8;
}

// Packed per-step constants of the pair sweep.
struct PairK {
    f2 dx, rdx, dd, rdd, w, A, invA, g, dt, rain, half, nmin, vcrK;
    f2 den, rden;                       // 2K dt and RN(1/(2K dt)) (volume cap)
    float tau_l, tau_h;
};

__device__ __forceinline__ f2 ld2(const float *p)
{
    const float2 v = __ldg(reinterpret_cast<const float2 *>(p));
    return mk2(v.x, v.y);
}
__device__ __forceinline__ f2 ld2_rw(const float *p)
{
    const float2 v = *reinterpret_cast<const float2 *>(p);
    return mk2(v.x, v.y);
}
__device__ __forceinline__ void st2(float *p, f2 v)
{
    *reinterpret_cast<float2 *>(p) = make_float2(lo2(v), hi2(v));
}
__device__ __forceinline__ f2 lds2(uint32_t a)
{
    float x, y;
    asm volatile("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(x), "=f"(y) : "r"(a));
    return mk2(x, y);
}

// RN(sqrt(g*hf)) per half of the exact product g*hf (as the reference's
// (real)sqrt((double)g*(double)hf), physics.h:107-108): from p = RN(g*hf),
// its error pe = g*hf - p (exact, one fused multiply-add) and s = RN(sqrt(p)),
// the root of p + pe is s + (p - s^2 + pe)/(2s) to far better than 2^-20 ulp;
// that sum is rounded to y with its error e (Fast2Sum). `unsure` per half:
// |e| within 2^-11 of half an ulp of y (tested as fma(e, 1 + 2^-11, y) != y),
// which also covers the reference's double rounding (its root is rounded to
// double first, which can only matter within 2^-29 ulp of a midpoint). The
// exact value is never a float midpoint: a midpoint has 25 significant bits,
// its square at least 49, and g*hf at most 48.
__device__ __forceinline__ f2 vcrit2(f2 g, f2 hf, bool &unsure0, bool &unsure1)
{
    const f2 p = mul2(g, hf);
    const f2 pe = fma2(g, hf, neg2(p));
    const f2 y0 = rsqrt_2(p);
    const f2 s0 = mul2(p, y0);
    const f2 h = mul2(bc2(0.5f), y0);
    const f2 s = fma2(fma2(neg2(s0), s0, p), h, s0);       // RN(sqrt(p))
    const f2 r = add2(fma2(neg2(s), s, p), pe);              // g*hf - s^2
    const f2 corr = mul2_sep(r, h);
    const f2 y = add2(s, corr);
    const f2 e = add2(sub2(s, y), corr);
    const f2 chk = fma2(e, bc2(1.00048828125f), y);
    float y0f, y1f, k0, k1;
    sp2(y, y0f, y1f);
    sp2(chk, k0, k1);
    unsure0 = k0 != y0f;
    unsure1 = k1 != y1f;
    return y;
}

// Discharge a -> b of two faces (one per half) between all-LAND cells with
// old levels La, Lb, elevations za, zb and Manning n na, nb, centre distance
// d (rd = RN(1/d)) and width w (FloodCA src/kernels/physics.h:51-125), with
// the critical-velocity and volume caps, in three parts so that the faces of
// a row run as one block of independent work: face2_v (the Manning velocity;
// `cr` flags live halves whose v may reach the critical velocity), then, in
// one branch for all faces of the row when any lane has such a half,
// face2_crit (v = min(v, RN(sqrt(g hf)))), then face2_q (discharge, volume
// cap). MATH_EXACT: every operation rounded as the reference's; `un` flags
// live halves whose value the exact scalar formula must settle (a cube root
// or critical velocity near a rounding midpoint, or out of range).
// MATH_FAST: hardware approximations throughout, no flags.
struct Face2 {
    f2 dL, adL, hf, v;
    bool live0, live1, cr0, cr1, un0, un1;
};

template <int MATH>
__device__ __forceinline__ Face2 face2_v(f2 La, f2 Lb, f2 za, f2 zb, f2 na, f2 nb, f2 d, f2 rd,
                                         const PairK &c)
{
    Face2 f;
    f.dL = sub2(La, Lb);
    const f2 Lmx = max2(La, Lb);
    f.adL = sub2(Lmx, min2(La, Lb));        // |dL|, the same rounding
    f.hf = sub2(Lmx, max2(za, zb));
    float a0, a1, h0, h1;
    sp2(f.adL, a0, a1);
    sp2(f.hf, h0, h1);
    f.live0 = a0 >= c.tau_l && h0 >= c.tau_h;
    f.live1 = a1 >= c.tau_l && h1 >= c.tau_h;
    const f2 nf = max2(mul2(c.half, add2(na, nb)), c.nmin);
    if constexpr (MATH == MATH_EXACT) {
        const f2 rnf = rcp2_nr(nf);
        const f2 sq = sqrt2_nr(div2_mk(f.adL, d, rd));
        bool s0, s1;
        const f2 cb = cbrt_sq2(f.hf, s0, s1);
        f.v = mul2(mul2(rnf, cb), sq);
        // v^2 < g hf (1 - 1e-6) leaves v surely below the critical velocity
        const f2 v2 = mul2(f.v, f.v);
        const f2 pm = mul2(mul2(c.g, f.hf), c.vcrK);
        f.cr0 = f.live0 && !(lo2(v2) < lo2(pm));
        f.cr1 = f.live1 && !(hi2(v2) < hi2(pm));
        f.un0 = f.live0 && s0;
        f.un1 = f.live1 && s1;
    } else {
        const f2 rnf = rcp_2(nf);
        const f2 S = mul2(f.adL, rd);
        const f2 sq = mul2(S, rsqrt_2(S));
        const f2 cb = ex2_2(mul2(lg2_2(f.hf), bc2(0.666666687f)));
        f2 v = mul2(mul2(rnf, cb), sq);
        const f2 p = mul2(c.g, f.hf);
        const f2 vcr = mul2(p, rsqrt_2(p));
        const f2 v2 = mul2(v, v);
        f.v = sel2(lo2(v2) > lo2(p), hi2(v2) > hi2(p), vcr, v);
        f.cr0 = f.cr1 = f.un0 = f.un1 = false;
    }
    return f;
}

// v = min(v, RN(sqrt(g hf))) on the flagged halves (exact mode)
__device__ __forceinline__ void face2_crit(Face2 &f, const PairK &c)
{
    bool vu0, vu1;
    const f2 vcr = vcrit2(c.g, f.hf, vu0, vu1);
    f.v = sel2(f.cr0, f.cr1, min2(f.v, vcr), f.v);
    f.un0 = f.un0 || (f.cr0 && vu0);
    f.un1 = f.un1 || (f.cr1 && vu1);
}

// Q = sign(dL) min(v hf w, RN(RN(|dL| A) / (2K dt))); cap: live halves
// whose volume cap binds
template <int MATH>
__device__ __forceinline__ f2 face2_q(const Face2 &f, f2 w, const PairK &c, bool &cap0,
                                      bool &cap1)
{
    const f2 Qm = mul2(mul2(f.v, f.hf), w);
    f2 Qc;
    if constexpr (MATH == MATH_EXACT)
        Qc = div2_mk(mul2(f.adL, c.A), c.den, c.rden);
    else
        Qc = mul2(mul2(f.adL, c.A), c.rden);
    cap0 = f.live0 && lo2(Qc) < lo2(Qm);
    cap1 = f.live1 && hi2(Qc) < hi2(Qm);
    const f2 Q = copysign2(min2(Qm, Qc), f.dL);
    return sel2(f.live0, f.live1, Q, bc2(0.0f));
}

// Exact re-evaluation of the flagged halves of a face pair with the scalar
// formula (face_q); `cap` counts the volume caps among them. The step
// constants come through a pointer (shared memory) so that no register of
// the caller has to live in memory around the call.
struct Settled {
    f2 Q;
    unsigned cap;
};

static __device__ __noinline__ Settled face2_settle(f2 Q, bool un0, bool un1, f2 za, f2 ha, f2 na,
                                                    f2 zb, f2 hb, f2 nb, bool diag,
                                                    const StepK<float> *kp)
{
    const StepK<float> k = *kp;
    const float d = diag ? k.d_diag : k.dx, rd = diag ? k.rdd : k.rdx;
    Settled o;
    o.cap = 0u;
#pragma unroll
    for (int j = 0; j < 2; j++) {
        if (j == 0 ? un0 : un1) {
            int cap = 0;
            const float q = face_q<float, MATH_EXACT>(get2(za, j), get2(ha, j), get2(na, j), M_LAND,
                                                      get2(zb, j), get2(hb, j), get2(nb, j), M_LAND,
                                                      d, rd, k, cap);
            put2(Q, j, q);
            o.cap += (unsigned)cap;
        }
    }
    o.Q = Q;
    return o;
}

// The exact next-step velocity of the flagged halves (physics.h:193-217),
// folded into the running maximum vm.
template <int K, int MATH>
__device__ __noinline__ float pair_velocity(float vm, bool x0, bool x1, f2 mo, f2 md, f2 hv, f2 nv,
                                            const StepK<float> *kp)
{
    const StepK<float> k = *kp;
#pragma unroll
    for (int j = 0; j < 2; j++) {
        if (j == 0 ? x0 : x1) {
            float Smax = Mth<float, MATH>::div(get2(mo, j), k.dx);
            if constexpr (K == 8) {
                const float Sd = Mth<float, MATH>::div(get2(md, j), k.d_diag);
                Smax = Sd > Smax ? Sd : Smax;
            }
            const float v = cell_velocity<float, MATH>(get2(hv, j), get2(nv, j), Smax, k);
            vm = v > vm ? v : vm;
        }
    }
    return vm;
}

// Open-edge faces of a row's two cells (model.c:442-479): discharge to the
// virtual neighbour, clipped at zero; `add` is what each cell adds to its
// outflow (the sum of its open slots, model.c:235-236), `ko` the open sides
// (4 bits per cell, one per side), `cap` the volume caps of owned cells.
struct OpenFaces {
    f2 qo, add;
    unsigned ko, cap;
};

static __device__ __noinline__ OpenFaces open_faces2(f2 z, f2 h, f2 n, int r, int cbase, int nr,
                                                     int nc, int r_lo, int r_hi, int edges,
                                                     bool own0, bool own1,
                                                     const StepK<float> *kp)
{
    const StepK<float> k = *kp;
    OpenFaces o;
    o.ko = 0u;
    o.cap = 0u;
    float q[2] = {0.0f, 0.0f}, a[2] = {0.0f, 0.0f};
#pragma unroll
    for (int j = 0; j < 2; j++) {
        const int cc = cbase + j;
        const bool inside = r >= r_lo && r < r_hi && cc >= 0 && cc < nc;
        // edges: bit 0 north, 1 south, 2 west, 3 east
        const int kop = inside ? (cc == 0 && (edges & 4)) + (cc == nc - 1 && (edges & 8)) +
                                     (r == 0 && (edges & 1)) + (r == nr - 1 && (edges & 2))
                               : 0;
        if (kop) {
            int cap;
            q[j] = open_q<float, MATH_EXACT>(get2(z, j), get2(h, j), get2(n, j), M_LAND, k, cap);
            if (j == 0 ? own0 : own1)
                o.cap += (unsigned)(cap * kop);
            a[j] = open_sum<float>(q[j], kop);
            o.ko |= (unsigned)((1 << kop) - 1) << (4 * j);
        }
    }
    o.qo = mk2(q[0], q[1]);
    o.add = mk2(a[0], a[1]);
    return o;
}

// The registers of the four-row ring (see the file comment).
template <int K>
struct PairRing {
    f2 z[4], h[4], n[4], L[4];          // row data, old level z + h
    f2 zr[4], hr[4], nr[4], Lr[4];      // right-shifted copies (K = 8 SW faces)
    f2 X[4];                            // x faces (c -> c+1) of a row
    f2 Y[4];                            // y faces (r -> r+1), by the upper row
    f2 E[4], W[4];                      // K = 8: SE (r,c)->(r+1,c+1), SW (r,c+1)->(r+1,c)
    f2 s[4];                            // limiter
    f2 Qy[4], Qe[4], Qw[4];             // scaled y / SE / SW discharges, by the upper row
    f2 Ln[4];                           // new level (NaN outside the grid)
    f2 cr[4];                           // rain field
    f2 qo[4];                           // open-edge discharge of edge cells
    unsigned ko[4];                     // open sides of the two cells (4 bits each)
    unsigned ef[4];                     // stage-E candidates (bit per half)
};

// Per-segment values of the pair sweep.
struct PairSeg {
    const float *gz, *gn, *hin, *gcr;
    float *hout, *ghmax, *gtmax;
    int pitch, colo;                    // 32-bit element offsets (grids checked on the host)
    int nr, nc, r0, r1, r_lo, r_hi;
    int cbase, edges;                   // open edges: bit 0 N, 1 S, 2 W, 3 E (0: closed)
    bool out_lane, edge_strip, col0ok, col1ok;
    float thr, thr2c, T6;               // stage-E thresholds (warp-uniform)
    // TMA row source
    const CUtensorMap *tz, *th, *tn;    // tensor maps of z, the input depth, n
    uint32_t ring, bars, srow;          // ring and barriers of the warp; next row's address
    uint32_t *phase;                    // barrier phase bits of the warp (persist over segments)
    int i0, blk, tx;                    // first row, current block, x of the strip
    bool tma_err;
    int o1;                             // element offset of row i+1 in the current iteration
};

// The ring viewed one row further: slot q takes slot q+1's registers.
template <typename V>
__device__ __forceinline__ void rot4(V (&a)[4])
{
    const V t = a[0];
    a[0] = a[1];
    a[1] = a[2];
    a[2] = a[3];
    a[3] = t;
}
// The ring viewed two rows further: slots q and q+2 swap.
template <typename V>
__device__ __forceinline__ void rot4x2(V (&a)[4])
{
    V t = a[0];
    a[0] = a[2];
    a[2] = t;
    t = a[1];
    a[1] = a[3];
    a[3] = t;
}
template <int K>
__device__ __forceinline__ void rotate_ring2(PairRing<K> &R)
{
    rot4x2(R.z); rot4x2(R.h); rot4x2(R.n); rot4x2(R.L);
    rot4x2(R.X); rot4x2(R.Y);
    rot4x2(R.s); rot4x2(R.Qy); rot4x2(R.Ln);
    rot4x2(R.cr); rot4x2(R.qo); rot4x2(R.ko); rot4x2(R.ef);
    if constexpr (K == 8) {
        rot4x2(R.zr); rot4x2(R.hr); rot4x2(R.nr); rot4x2(R.Lr);
        rot4x2(R.E); rot4x2(R.W);
        rot4x2(R.Qe); rot4x2(R.Qw);
    }
}
template <int K>
__device__ __forceinline__ void rotate_ring(PairRing<K> &R)
{
    rot4(R.z); rot4(R.h); rot4(R.n); rot4(R.L);
    rot4(R.X); rot4(R.Y);
    rot4(R.s); rot4(R.Qy); rot4(R.Ln);
    rot4(R.cr); rot4(R.qo); rot4(R.ko); rot4(R.ef);
    if constexpr (K == 8) {
        rot4(R.zr); rot4(R.hr); rot4(R.nr); rot4(R.Lr);
        rot4(R.E); rot4(R.W);
        rot4(R.Qe); rot4(R.Qw);
    }
}

template <typename AccT, int K, int MATH, bool RAINF>
struct PairSweep {
    using SS = StepSums<float, AccT>;

    // ---- TMA row source
    // lane 0: block b (rows i0 + 8b .. +7) of z, h, n into stage b % TMA_NS
    static __device__ __forceinline__ void tma_issue(const PairSeg &G, int b)
    {
        const int st = b % TMA_NS;
        const uint32_t bar = G.bars + 8u * st, dst = G.ring + st * TMA_STAGE_B;
        const int y = G.i0 + b * TMA_RB + PADR;
        mbar_arrive_tx(bar, TMA_STAGE_B);
        tma_load_tile(dst, G.tz, bar, G.tx, y);
        tma_load_tile(dst + TMA_FIELD_B, G.th, bar, G.tx, y);
        tma_load_tile(dst + 2 * TMA_FIELD_B, G.tn, bar, G.tx, y);
    }
    static __device__ __forceinline__ void tma_wait(PairSeg &G, int b)
    {
        const int st = b % TMA_NS;
        if (!mbar_wait_bounded(G.bars + 8u * st, (*G.phase >> st) & 1u))
            G.tma_err = true;
        *G.phase ^= 1u << st;
    }
    // moves to block b: refills the stage of block b-1 (all lanes are past
    // it) with block b + TMA_NS - 1, then waits for block b
    static __device__ __forceinline__ void tma_turn(PairSeg &G, int lane)
    {
        const int b = ++G.blk;
        __syncwarp();
        if (lane == 0) {
            fence_proxy_async_smem();
            tma_issue(G, b + TMA_NS - 1);
        }
        tma_wait(G, b);
        G.srow = G.ring + (b % TMA_NS) * TMA_STAGE_B + lane * 8;
    }

    // thr = max(warp maximum so far, seed); thr2c = thr^2 (1 - 1e-6) for the
    // critical-velocity prefilter; T6 = thr^6 (1 - 2e-4) for the bound (0 when
    // thr < 1e-6: every velocity is at least 1e-6, physics.h:214-216)
    static __device__ __forceinline__ void thresholds(PairSeg &G, float wmax, float vseed)
    {
        const float thr = wmax > vseed ? wmax : vseed;
        G.thr = thr;
        G.thr2c = thr * thr * 0.999999f;
        const float t2 = thr * thr;
        G.T6 = thr >= 1e-6f ? t2 * t2 * t2 * 0.9998f : 0.0f;
    }

    // one iteration of the pipeline; J = (i - i0) & 3
    template <int J, bool TMA>
    static __device__ __forceinline__ void iter(PairRing<K> &R, PairSeg &G, const PairK &c,
                                                const StepVals<float> &sv, const RunK<float> &rk,
                                                const StepK<float> *kp, SS &ss, int i, int lane)
    {
        constexpr int S1 = (J + 1) & 3;   // row i+1
        constexpr int S0 = J & 3;         // row i
        constexpr int Sm1 = (J + 3) & 3;  // row i-1
        constexpr int Sm2 = (J + 2) & 3;  // row i-2
        constexpr int Sm3 = (J + 1) & 3;  // row i-3
        constexpr int Sm4 = J & 3;        // row i-4
        const int pitch = G.pitch;
        const f2 z0 = bc2(0.0f);
        f2 hm_i2;                         // hmax of row i-2 (stage D)

        // ---- loads: row i+1, the rain field of row i-1, hmax of row i-2
        {
            const int off = G.o1;
            G.o1 += pitch;
            if constexpr (TMA) {
                // row i+1 is row i+1-i0 of the stream: a new block every 8
                // rows, which (8 being a multiple of the rows per pass) a
                // pass only meets in its last iteration
                if ((FCAB_PAIR_UNROLL == 1 || J == FCAB_PAIR_UNROLL - 1) &&
                    ((i + 1 - G.i0) & (TMA_RB - 1)) == 0)
                    tma_turn(G, lane);
                R.z[S1] = lds2(G.srow);
                R.h[S1] = lds2(G.srow + TMA_FIELD_B);
                R.n[S1] = lds2(G.srow + 2 * TMA_FIELD_B);
                G.srow += 256;
            } else {
                R.z[S1] = ld2(G.gz + off);
                R.h[S1] = ld2(G.hin + off);
                R.n[S1] = ld2(G.gn + off);
                const int offa = i + 1 + PF_ROWS <= G.nr + PADR - 1
                                     ? off + PF_ROWS * pitch
                                     : (G.nr + 2 * PADR - 1) * pitch + G.colo;
                prefetch_l2(G.gz + offa);
                prefetch_l2(G.hin + offa);
                prefetch_l2(G.gn + offa);
            }
            const int off1 = off - 2 * pitch;
            // hmax of row i-2, loaded in the iteration that updates it: a
            // ring slot carried from the row before held two more registers
            // through the rotation and ran 0.7 % slower at 16 warps
            hm_i2 = G.out_lane && i - 2 >= G.r0 && i - 2 < G.r1 ? ld2_rw(G.ghmax + off - 3 * pitch) : z0;
            // every ring slot is written on every row, so no register of an
            // older row stays live through the rotation
            if constexpr (RAINF)
                R.cr[Sm1] = ld2(G.gcr + off1);
        }

        // ---- A: x faces of row i; y (and diagonal) faces between rows i-1 and i
        {
            R.L[S0] = add2(R.z[S0], R.h[S0]);
            const f2 zr = right2(R.z[S0]), Lr = right2(R.L[S0]), nrr = right2(R.n[S0]);
            Face2 fx = face2_v<MATH>(R.L[S0], Lr, R.z[S0], zr, R.n[S0], nrr, c.dx, c.rdx, c);
            Face2 fy = face2_v<MATH>(R.L[Sm1], R.L[S0], R.z[Sm1], R.z[S0], R.n[Sm1], R.n[S0], c.dx,
                                     c.rdx, c);
            Face2 fe, fw;
            if constexpr (K == 8) {
                R.zr[S0] = zr;
                R.Lr[S0] = Lr;
                R.nr[S0] = nrr;
                fe = face2_v<MATH>(R.L[Sm1], Lr, R.z[Sm1], zr, R.n[Sm1], nrr, c.dd, c.rdd, c);
                fw = face2_v<MATH>(R.Lr[Sm1], R.L[S0], R.zr[Sm1], R.z[S0], R.nr[Sm1], R.n[S0], c.dd,
                                   c.rdd, c);
            }
            if constexpr (MATH == MATH_EXACT) {
                bool crit = fx.cr0 || fx.cr1 || fy.cr0 || fy.cr1;
                if constexpr (K == 8)
                    crit = crit || fe.cr0 || fe.cr1 || fw.cr0 || fw.cr1;
                if (__any_sync(0xffffffffu, crit)) {
                    face2_crit(fx, c);
                    face2_crit(fy, c);
                    if constexpr (K == 8) {
                        face2_crit(fe, c);
                        face2_crit(fw, c);
                    }
                }
            }
            bool cx0, cx1, cy0, cy1;
            f2 X = face2_q<MATH>(fx, c.w, c, cx0, cx1);
            f2 Y = face2_q<MATH>(fy, c.w, c, cy0, cy1);
            const bool ux0 = fx.un0, ux1 = fx.un1, uy0 = fy.un0, uy1 = fy.un1;
            f2 E = z0, W = z0;
            bool ue0 = false, ue1 = false, uw0 = false, uw1 = false;
            bool ce0 = false, ce1 = false, cw0 = false, cw1 = false;
            if constexpr (K == 8) {
                E = face2_q<MATH>(fe, c.w, c, ce0, ce1);
                W = face2_q<MATH>(fw, c.w, c, cw0, cw1);
                ue0 = fe.un0;
                ue1 = fe.un1;
                uw0 = fw.un0;
                uw1 = fw.un1;
            }
            // faces are counted by the cell that holds them: x faces by row i,
            // y and diagonal faces by row i-1; volume caps of the halves the
            // exact re-evaluation does not redo
            const bool ownA = G.out_lane && i >= G.r0 && i < G.r1;
            const bool ownB = G.out_lane && i - 1 >= G.r0 && i - 1 < G.r1;
            if (ownA)
                ss.capn += (unsigned)(cx0 && !ux0) + (unsigned)(cx1 && !ux1);
            if (ownB) {
                ss.capn += (unsigned)(cy0 && !uy0) + (unsigned)(cy1 && !uy1);
                if constexpr (K == 8)
                    ss.capn += (unsigned)(ce0 && !ue0) + (unsigned)(ce1 && !ue1) +
                               (unsigned)(cw0 && !uw0) + (unsigned)(cw1 && !uw1);
            }
            if constexpr (MATH == MATH_EXACT) {
                bool any = ux0 || ux1 || uy0 || uy1;
                if constexpr (K == 8)
                    any = any || ue0 || ue1 || uw0 || uw1;
                const bool settle = __any_sync(0xffffffffu, any);
                f2 hr = z0;
                if (K == 8 || settle)
                    hr = right2(R.h[S0]);
                if constexpr (K == 8)
                    R.hr[S0] = hr;
                if (settle) {
                    if (ux0 || ux1) {
                        const Settled o = face2_settle(X, ux0, ux1, R.z[S0], R.h[S0], R.n[S0], zr,
                                                       hr, nrr, false, kp);
                        X = o.Q;
                        if (ownA)
                            ss.capn += o.cap;
                    }
                    if (uy0 || uy1) {
                        const Settled o = face2_settle(Y, uy0, uy1, R.z[Sm1], R.h[Sm1], R.n[Sm1],
                                                       R.z[S0], R.h[S0], R.n[S0], false, kp);
                        Y = o.Q;
                        if (ownB)
                            ss.capn += o.cap;
                    }
                    if constexpr (K == 8) {
                        if (ue0 || ue1) {
                            const Settled o = face2_settle(E, ue0, ue1, R.z[Sm1], R.h[Sm1],
                                                           R.n[Sm1], zr, hr, nrr, true, kp);
                            E = o.Q;
                            if (ownB)
                                ss.capn += o.cap;
                        }
                        if (uw0 || uw1) {
                            const Settled o = face2_settle(W, uw0, uw1, R.zr[Sm1], R.hr[Sm1],
                                                           R.nr[Sm1], R.z[S0], R.h[S0], R.n[S0],
                                                           true, kp);
                            W = o.Q;
                            if (ownB)
                                ss.capn += o.cap;
                        }
                    }
                }
            }
            R.X[S0] = X;
            R.Y[Sm1] = Y;
            if constexpr (K == 8) {
                R.E[Sm1] = E;
                R.W[Sm1] = W;
            }
        }

        // ---- C: outflow volume and limiter of row i-1 (model.c:180-238,
        //      489-502), in the reference order +x, -x, +y, -y, d1+, d1-,
        //      d2+, d2-, open slots
        {
            const int r = i - 1;
            // max(Q, 0) of the faces leaving, -min(Q, 0) of the faces entering
            f2 out = sub2(max2(R.X[Sm1], z0), min2(left2(R.X[Sm1]), z0));
            out = add2(out, max2(R.Y[Sm1], z0));
            out = sub2(out, min2(R.Y[Sm2], z0));
            if constexpr (K == 8) {
                out = add2(out, max2(R.E[Sm1], z0));
                out = sub2(out, min2(left2(R.E[Sm2]), z0));
                out = add2(out, max2(left2(R.W[Sm1]), z0));
                out = sub2(out, min2(R.W[Sm2], z0));
            }
            R.ko[Sm1] = 0u;
            R.qo[Sm1] = z0;
            if (G.edges) {
                const bool erow = (r == 0 && (G.edges & 1)) || (r == G.nr - 1 && (G.edges & 2));
                if (erow || G.edge_strip) {
                    const bool own = G.out_lane && r >= G.r0 && r < G.r1;
                    const OpenFaces o = open_faces2(R.z[Sm1], R.h[Sm1], R.n[Sm1], r, G.cbase,
                                                    G.nr, G.nc, G.r_lo, G.r_hi, G.edges,
                                                    own && G.col0ok, own && G.col1ok, kp);
                    R.ko[Sm1] = o.ko;
                    R.qo[Sm1] = o.qo;
                    ss.capn += o.cap;
                    out = add2(out, o.add);
                }
            }
            const f2 ov = mul2(out, c.dt);
            const f2 hold = mul2(R.h[Sm1], c.A);
            const f2 hz = max2(hold, z0);
            const bool l0 = lo2(ov) > lo2(hz), l1 = hi2(ov) > hi2(hz);
            R.s[Sm1] = bc2(1.0f);
            if (__any_sync(0xffffffffu, l0 || l1)) {
                const f2 o = sel2(l0, l1, ov, bc2(1.0f));
                f2 q;
                if constexpr (MATH == MATH_EXACT)
                    q = div2_mk(hold, o, rcp2_nr(o));
                else
                    q = mul2(hold, rcp_2(o));
                R.s[Sm1] = sel2(l0, l1, q, bc2(1.0f));
            }
        }

        // ---- D: scaled discharges of the faces below and right of row i-2,
        //      net inflow, depth update, clamp, inflow, hmax/tmax, stage-E
        //      candidates (model.c:511-597)
        {
            const int r = i - 2;
            const bool row_out = r >= G.r0 && r < G.r1;
            const f2 s0 = R.s[Sm2];
            const f2 sr = right2(s0);
            const f2 Qsx = fma2(min2(R.X[Sm2], z0), sr, mul2(max2(R.X[Sm2], z0), s0));
            const f2 Qsy = fma2(min2(R.Y[Sm2], z0), R.s[Sm1], mul2(max2(R.Y[Sm2], z0), s0));
            R.Qy[Sm2] = Qsy;
            f2 net = sub2(z0, Qsx);
            net = add2(net, left2(Qsx));
            net = sub2(net, Qsy);
            net = add2(net, R.Qy[Sm3]);
            if constexpr (K == 8) {
                const f2 Qse = fma2(min2(R.E[Sm2], z0), right2(R.s[Sm1]),
                                    mul2(max2(R.E[Sm2], z0), s0));
                const f2 Qsw = fma2(min2(R.W[Sm2], z0), R.s[Sm1], mul2(max2(R.W[Sm2], z0), sr));
                R.Qe[Sm2] = Qse;
                R.Qw[Sm2] = Qsw;
                net = sub2(net, Qse);
                net = add2(net, left2(R.Qe[Sm3]));
                net = sub2(net, left2(Qsw));
                net = add2(net, R.Qw[Sm3]);
            }
            const bool cell0 = row_out && G.out_lane && G.col0ok;
            const bool cell1 = row_out && G.out_lane && G.col1ok;
            if (G.edges && __any_sync(0xffffffffu, R.ko[Sm2] != 0u)) {
                // open-edge outflow scaled by the cell's own limiter
                // (model.c:553-559), summed over its open slots
                float qb[2];
#pragma unroll
                for (int j = 0; j < 2; j++) {
                    const unsigned kk = (R.ko[Sm2] >> (4 * j)) & 15u;
                    qb[j] = open_sum<float>(get2(R.qo[Sm2], j) * get2(s0, j), __popc(kk));
                }
                net = sub2(net, mk2(qb[0], qb[1]));
                if (cell0 && (R.ko[Sm2] & 15u))
                    ss.a_bnd += acc_mul<AccT, float>(sv.dt, qb[0]);
                if (cell1 && (R.ko[Sm2] >> 4))
                    ss.a_bnd += acc_mul<AccT, float>(sv.dt, qb[1]);
            }
            f2 rain = c.rain;
            if constexpr (RAINF)
                rain = mul2_sep(R.cr[Sm2], bc2(sv.F));
            f2 dq;
            if constexpr (MATH == MATH_EXACT)
                dq = div2_mk(net, c.A, c.invA);
            else
                dq = mul2(net, c.invA);
            f2 hu = add2(R.h[Sm2], add2(mul2_sep(c.dt, dq), rain));
            {
                float u0, u1;
                sp2(hu, u0, u1);
                if (__any_sync(0xffffffffu, u0 < 0.0f || u1 < 0.0f)) {
                    if (u0 < 0.0f) {
                        if (cell0)
                            ss.a_clamp += acc_mul<AccT, float>(-u0, sv.A);
                        u0 = 0.0f;
                    }
                    if (u1 < 0.0f) {
                        if (cell1)
                            ss.a_clamp += acc_mul<AccT, float>(-u1, sv.A);
                        u1 = 0.0f;
                    }
                    hu = mk2(u0, u1);
                }
            }
            if (r == rk.inflow_r) {
                const int d = rk.inflow_c - G.cbase;
                if (d == 0)
                    hu = mk2(lo2(hu) + sv.inflow_dh, hi2(hu));
                else if (d == 1)
                    hu = mk2(lo2(hu), hi2(hu) + sv.inflow_dh);
            }
            if constexpr (sizeof(AccT) == 4) {
                if (cell0)
                    ss.a_rain += sv.A * lo2(rain);
                if (cell1)
                    ss.a_rain += sv.A * hi2(rain);
            } else if constexpr (RAINF) {
                ss.rain_sum += (cell0 ? (double)lo2(rain) : 0.0) + (cell1 ? (double)hi2(rain) : 0.0);
            }
            // new level for stage E (NaN outside the grid: no neighbour
            // there); cells outside the grid keep their padding depth
            f2 Ln = add2(R.z[Sm2], hu);
            f2 hkeep = hu;
            if (G.edge_strip || r < G.r_lo || r >= G.r_hi) {
                const bool rin = r >= G.r_lo && r < G.r_hi;
                const bool in0 = rin && G.col0ok, in1 = rin && G.col1ok;
                Ln = sel2(in0, in1, Ln, bc2(__int_as_float(0x7fc00000)));
                hkeep = sel2(in0, in1, hu, R.h[Sm2]);
            }
            R.Ln[Sm2] = Ln;
            // stage-E candidates: wet output cells whose critical velocity
            // sqrt(g h) may exceed the warp's threshold (margin 1e-6)
            unsigned ef = 0u;
            if (sv.want_v) {
                const f2 gh = mul2(c.g, hu);
                const bool t = G.thr > 0.0f;
                if (cell0 && lo2(hu) >= c.tau_h && !(t && lo2(gh) <= G.thr2c))
                    ef |= 1u;
                if (cell1 && hi2(hu) >= c.tau_h && !(t && hi2(gh) <= G.thr2c))
                    ef |= 2u;
            }
            R.ef[Sm2] = ef;
            // hmax / tmax of output cells
            const f2 hmo = hm_i2;
            const bool rise0 = cell0 && lo2(hu) > lo2(hmo);
            const bool rise1 = cell1 && hi2(hu) > hi2(hmo);
            if (row_out && G.out_lane) {
                // hmax is written back whether or not it rose (no divergent
                // branch; the loaded value where it did not), tmax where it rose
                const int off2 = G.o1 - 4 * pitch;              // row i-2
                st2(G.hout + off2, hkeep);
                st2(G.ghmax + off2, sel2(rise0, rise1, hu, hmo));
                if (rise0)
                    G.gtmax[off2] = sv.tmax_val;
                if (rise1)
                    G.gtmax[off2 + 1] = sv.tmax_val;
            }
        }

        // ---- E: next step's stable velocity of row i-3 from the new levels
        //      of rows i-4..i-2 (physics.h:158-217), for the candidates
        if (sv.want_v && __any_sync(0xffffffffu, R.ef[Sm3] != 0u)) {
            const int r = i - 3;
            const f2 la = R.Ln[Sm3];
            f2 mo = max2(abs2(sub2(la, right2(la))), abs2(sub2(la, left2(la))));
            mo = max2(mo, max2(abs2(sub2(la, R.Ln[Sm2])), abs2(sub2(la, R.Ln[Sm4]))));
            mo = max2(mo, z0);
            f2 md = z0;
            if constexpr (K == 8) {
                const f2 lb = R.Ln[Sm2], lt = R.Ln[Sm4];
                md = max2(abs2(sub2(la, right2(lb))), abs2(sub2(la, left2(lb))));
                md = max2(md, max2(abs2(sub2(la, right2(lt))), abs2(sub2(la, left2(lt)))));
                md = max2(md, z0);
            }
            if (G.edges) {
                const bool erow = (r == 0 && (G.edges & 1)) || (r == G.nr - 1 && (G.edges & 2));
                if (erow || G.edge_strip) {
                    // the open virtual neighbour z - S_bnd*dx, h = 0 (physics.h:183-189)
                    const int off3 = G.o1 - 5 * pitch;          // row i-3
                    const f2 z3 = ld2(G.gz + off3);
                    const f2 dv = abs2(sub2(la, sub2(z3, bc2(sv.k.S_bnd * sv.k.dx))));
#pragma unroll
                    for (int j = 0; j < 2; j++) {
                        const int cc = G.cbase + j;
                        if (erow || (cc == 0 && (G.edges & 4)) || (cc == G.nc - 1 && (G.edges & 8)))
                            put2(mo, j, fmaxf(get2(mo, j), get2(dv, j)));
                    }
                }
            }
            // bound: v^6 <= h^4 S^3 / n^6 (S = the largest slope), against thr^6.
            // n and the new depth are read here, in the rare body, rather
            // than carried in the ring through every row: a candidate is an
            // output cell, whose new depth this thread stored in stage D of
            // the previous row (the coherent load sees it); other lanes load
            // nothing
            const int off3 = G.o1 - 5 * pitch;                  // row i-3
            const unsigned ef = R.ef[Sm3];
            const f2 n3 = ld2(G.gn + off3);
            const f2 n2 = mul2(n3, n3);
            f2 S = mul2(mo, c.rdx);
            if constexpr (K == 8)
                S = max2(S, mul2(md, c.rdd));
            const f2 hv = ef != 0u ? ld2_rw(G.hout + off3) : z0;
            const f2 h2 = mul2(hv, hv);
            const f2 lhs = mul2(mul2(h2, h2), mul2(mul2(S, S), S));
            const f2 rhs = mul2(mul2(mul2(n2, n2), n2), bc2(G.T6));
            const bool x0 = (ef & 1u) && (lo2(lhs) >= lo2(rhs) || lo2(lhs) < 1e-30f);
            const bool x1 = (ef & 2u) && (hi2(lhs) >= hi2(rhs) || hi2(lhs) < 1e-30f);
            if (__any_sync(0xffffffffu, x0 || x1)) {
                float vm = ss.vmax;
                if (x0 || x1)
                    vm = pair_velocity<K, MATH>(vm, x0, x1, mo, md, hv, n3, kp);
                ss.vmax = vm;
                thresholds(G, warp_max_nonneg(vm), sv.vseed);
            }
        }
    }

    // One warp streams output rows [r0, r1) of one strip (as sweep_segment).
    // kp: the step constants in shared memory, for the exact re-evaluations;
    // ring, bars, phase: the warp's TMA ring, barriers and phase bits (the
    // rows come by TMA when the grid has tensor maps, else by plain loads).
    static __device__ __forceinline__ void run(const GridD<float> &g, const RunK<float> &rk,
                               const StepVals<float> &sv, const StepK<float> *kp, int strip, int r0,
                               int r1, int lane, SS &ss, uint32_t ring = 0u, uint32_t bars = 0u,
                               uint32_t *phase = nullptr, bool *tma_err = nullptr)
    {
        if (g.tmap && ring)
            run_impl<true>(g, rk, sv, kp, strip, r0, r1, lane, ss, ring, bars, phase, tma_err);
        else
            run_impl<false>(g, rk, sv, kp, strip, r0, r1, lane, ss, 0u, 0u, nullptr, nullptr);
    }

    template <bool TMA>
    static __device__ __forceinline__ void run_impl(const GridD<float> &g, const RunK<float> &rk,
                                    const StepVals<float> &sv, const StepK<float> *kp, int strip,
                                    int r0, int r1, int lane, SS &ss, uint32_t ring, uint32_t bars,
                                    uint32_t *phase, bool *tma_err)
    {
        using Gm = Geom<2>;
        PairSeg G;
        G.gz = g.z;
        G.gn = g.n;
        G.gcr = g.cr;
        G.hin = sv.hin;
        G.hout = sv.hout;
        G.ghmax = g.hmax;
        G.gtmax = g.tmax;
        G.pitch = (int)g.pitch;
        G.nr = g.nr;
        G.nc = g.nc;
        G.r0 = r0;
        G.r1 = r1;
        G.r_lo = g.r_lo;
        G.r_hi = g.r_hi;
        G.cbase = strip * Gm::OW - Gm::HL + lane * 2;
        G.colo = G.cbase + PADC;
        G.out_lane = lane * 2 >= Gm::HL && lane * 2 < Gm::HL + Gm::OW;
        G.col0ok = G.cbase >= 0 && G.cbase < g.nc;
        G.col1ok = G.cbase + 1 >= 0 && G.cbase + 1 < g.nc;
        G.edges = rk.open ? (rk.edge_n ? 1 : 0) | (rk.edge_s ? 2 : 0) | (rk.edge_w ? 4 : 0) |
                                (rk.edge_e ? 8 : 0)
                          : 0;
        // strips that hold a column outside the grid or column 0 / nc-1
        const int c_first = strip * Gm::OW - Gm::HL;
        G.edge_strip = c_first <= 0 || c_first + Gm::SW > g.nc - 1;
        thresholds(G, sv.want_v ? warp_max_nonneg(ss.vmax) : 0.0f, sv.vseed);

        const StepK<float> &k = sv.k;
        PairK c;
        c.dx = bc2(k.dx);
        c.rdx = bc2(k.rdx);
        c.dd = bc2(k.d_diag);
        c.rdd = bc2(k.rdd);
        c.w = bc2(k.w);
        c.A = bc2(k.A);
        c.invA = bc2(k.inv_A);
        c.g = bc2(k.g);
        c.dt = bc2(sv.dt);
        c.rain = bc2(sv.rainv);
        c.half = bc2(0.5f);
        c.nmin = bc2(1e-12f);
        c.vcrK = bc2(0.99999905f);
        c.den = bc2(k.den);
        c.rden = bc2(k.rden);
        c.tau_l = k.tau_l;
        c.tau_h = k.tau_h;

        // iterations i0 .. r1+2, a multiple of four; the extra leading
        // iterations compute rows above the segment's halo only
        const int n_it = ((r1 - r0 + 6) + 3) & ~3;
        const int i0 = r1 + 3 - n_it;
        G.i0 = i0;
        G.tma_err = false;

        PairRing<K> R;
        const f2 z0 = bc2(0.0f);
#pragma unroll
        for (int q = 0; q < 4; q++) {
            R.z[q] = R.h[q] = R.n[q] = R.L[q] = z0;
            R.zr[q] = R.hr[q] = R.nr[q] = R.Lr[q] = z0;
            R.X[q] = R.Y[q] = R.E[q] = R.W[q] = z0;
            R.s[q] = bc2(1.0f);
            R.Qy[q] = R.Qe[q] = R.Qw[q] = z0;
            R.cr[q] = R.qo[q] = z0;
            R.Ln[q] = bc2(__int_as_float(0x7fc00000));
            R.ko[q] = R.ef[q] = 0u;
        }
        if constexpr (TMA) {
            G.tz = g.tmap;
            G.tn = g.tmap + 1;
            G.th = g.tmap + (sv.hin == g.h1 ? 3 : 2);
            G.ring = ring;
            G.bars = bars;
            G.phase = phase;
            G.tx = strip * Gm::OW - Gm::HL + PADC;      // a multiple of 4 floats
            G.blk = 0;
            __syncwarp();
            if (lane == 0) {
                fence_proxy_async_smem();
                for (int b = 0; b < TMA_NS; b++)
                    tma_issue(G, b);
            }
            tma_wait(G, 0);
            G.srow = G.ring + lane * 8;
            R.z[0] = lds2(G.srow);
            R.h[0] = lds2(G.srow + TMA_FIELD_B);
            R.n[0] = lds2(G.srow + 2 * TMA_FIELD_B);
            G.srow += 256;
        } else {
            const int off = (i0 + PADR) * G.pitch + G.colo;
            R.z[0] = ld2(G.gz + off);
            R.h[0] = ld2(G.hin + off);
            R.n[0] = ld2(G.gn + off);
        }
        G.o1 = (i0 + 1 + PADR) * G.pitch + G.colo;
        if constexpr (FCAB_PAIR_UNROLL == 1) {
            for (int i = i0; i < i0 + n_it; i++) {
                iter<0, TMA>(R, G, c, sv, rk, kp, ss, i, lane);
                rotate_ring<K>(R);
            }
        } else if constexpr (FCAB_PAIR_UNROLL == 2) {
            for (int i = i0; i < i0 + n_it; i += 2) {
                iter<0, TMA>(R, G, c, sv, rk, kp, ss, i, lane);
                iter<1, TMA>(R, G, c, sv, rk, kp, ss, i + 1, lane);
                rotate_ring2<K>(R);
            }
        } else {
            for (int i = i0; i < i0 + n_it; i += 4) {
                iter<0, TMA>(R, G, c, sv, rk, kp, ss, i, lane);
                iter<1, TMA>(R, G, c, sv, rk, kp, ss, i + 1, lane);
                iter<2, TMA>(R, G, c, sv, rk, kp, ss, i + 2, lane);
                iter<3, TMA>(R, G, c, sv, rk, kp, ss, i + 3, lane);
            }
        }
        if constexpr (TMA) {
            // no load may still be writing the ring when the next segment
            // starts: wait for the blocks issued ahead
            for (int b = G.blk + 1; b < G.blk + TMA_NS; b++)
                tma_wait(G, b);
            __syncwarp();
            if (G.tma_err && tma_err)
                *tma_err = true;
        }
        // uniform rain on LAND output cells, counted per lane
        if constexpr (sizeof(AccT) == 8 && !RAINF) {
            if (G.out_lane)
                ss.rain_cells += (long long)(r1 - r0) * ((G.col0ok ? 1 : 0) + (G.col1ok ? 1 : 0));
        }
    }
};

}  // namespace fcab
