// The FP32 sweep on four columns per lane for all-LAND grids with K = 4.
//
// The pair sweep's pipeline (wca_sweep_f2.cuh: iteration i loads row i+1 and
// runs A faces of rows i-1/i, C limiter of row i-1, D update of row i-2, E
// next-step velocity of row i-3; FloodCA src/kernels/physics.h and
// src/common/model.c:321-605) with each lane holding two column pairs
// (columns 4l .. 4l+3 of its strip) instead of one. Every per-pair formula
// is the pair sweep's own (face2_v, face2_crit, face2_q, face2_settle,
// open_faces2, pair_velocity), applied to both pairs; what changes is the
// neighbour exchange (the right neighbour of the first pair is in the same
// lane, only the outer columns cross lanes) and the strip geometry (128
// columns, 120 written). A lane's row tests, branches, votes and address
// arithmetic are shared by four cells instead of two, and the strip halo is
// 8 of 128 columns instead of 8 of 64.
#pragma once

#include "wca_sweep_f2.cuh"

namespace fcab {

// Two column pairs of a lane: p[0] columns 4l, 4l+1; p[1] columns 4l+2, 4l+3.
struct f4 {
    f2 p[2];
};

__device__ __forceinline__ f4 bc4(float a)
{
    f4 r;
    r.p[0] = r.p[1] = bc2(a);
    return r;
}
#define FCAB_F4_BINOP(name, op)                                                 \
    __device__ __forceinline__ f4 name(f4 a, f4 b)                             \
    {                                                                          \
        f4 r;                                                                  \
        r.p[0] = op(a.p[0], b.p[0]);                                           \
        r.p[1] = op(a.p[1], b.p[1]);                                           \
        return r;                                                              \
    }
FCAB_F4_BINOP(add4, add2)
FCAB_F4_BINOP(sub4, sub2)
FCAB_F4_BINOP(max4, max2)
FCAB_F4_BINOP(min4, min2)
#undef FCAB_F4_BINOP

// Columns c+1 of the lane's four columns (column 4l+4 from the next lane).
__device__ __forceinline__ f4 right4(f4 v)
{
    f4 r;
    r.p[0] = mk2(hi2(v.p[0]), lo2(v.p[1]));
    r.p[1] = mk2(hi2(v.p[1]), __shfl_down_sync(0xffffffffu, lo2(v.p[0]), 1));
    return r;
}
// Columns c-1 (column 4l-1 from the previous lane).
__device__ __forceinline__ f4 left4(f4 v)
{
    f4 r;
    r.p[0] = mk2(__shfl_up_sync(0xffffffffu, hi2(v.p[1]), 1), lo2(v.p[0]));
    r.p[1] = mk2(hi2(v.p[0]), lo2(v.p[1]));
    return r;
}

__device__ __forceinline__ f4 ld4(const float *p)
{
    const float4 v = __ldg(reinterpret_cast<const float4 *>(p));
    f4 r;
    r.p[0] = mk2(v.x, v.y);
    r.p[1] = mk2(v.z, v.w);
    return r;
}
__device__ __forceinline__ f4 ld4_rw(const float *p)
{
    const float4 v = *reinterpret_cast<const float4 *>(p);
    f4 r;
    r.p[0] = mk2(v.x, v.y);
    r.p[1] = mk2(v.z, v.w);
    return r;
}
__device__ __forceinline__ void st4(float *p, f4 v)
{
    *reinterpret_cast<float4 *>(p) =
        make_float4(lo2(v.p[0]), hi2(v.p[0]), lo2(v.p[1]), hi2(v.p[1]));
}
// half j (0..3) of the lane's four columns
__device__ __forceinline__ float get4(f4 v, int j) { return get2(v.p[j >> 1], j & 1); }

// The registers of the four-row ring (K = 4).
struct QuadRing {
    f4 z[4], h[4], n[4], L[4];          // row data, old level z + h
    f4 X[4], Y[4];                      // x faces (c -> c+1), y faces (r -> r+1) by the upper row
    f4 s[4], Qy[4];                     // limiter, scaled y discharge by the upper row
    f4 hn[4], Ln[4], n6[4];             // new depth, new level (NaN outside the grid), n^6
    f4 hm[4], cr[4], qo[4];             // hmax, rain field, open-edge discharge
    unsigned ko[4];                     // open sides of the four cells (4 bits each)
    unsigned ef[4];                     // stage-E candidates (bit per cell)
};

// Per-segment values of the four-column sweep.
struct QuadSeg {
    const float *gz, *gn, *hin, *gcr;
    float *hout, *ghmax, *gtmax;
    int pitch, colo, o1;                // 32-bit element offsets (grids checked on the host)
    int nr, nc, r0, r1, r_lo, r_hi;
    int cbase, edges;                   // open edges: bit 0 N, 1 S, 2 W, 3 E (0: closed)
    bool out_lane, edge_strip;
    unsigned colok;                     // bit j: column cbase + j inside the grid
    float thr, thr2c, T6;               // stage-E thresholds (warp-uniform)
};

template <typename V>
__device__ __forceinline__ void rot4q(V (&a)[4])
{
    const V t = a[0];
    a[0] = a[1];
    a[1] = a[2];
    a[2] = a[3];
    a[3] = t;
}
__device__ __forceinline__ void rotate_quad(QuadRing &R)
{
    rot4q(R.z); rot4q(R.h); rot4q(R.n); rot4q(R.L);
    rot4q(R.X); rot4q(R.Y); rot4q(R.s); rot4q(R.Qy);
    rot4q(R.hn); rot4q(R.Ln); rot4q(R.n6);
    rot4q(R.hm); rot4q(R.cr); rot4q(R.qo); rot4q(R.ko); rot4q(R.ef);
}

__device__ __forceinline__ f2 abs2d(f2 a, f2 b) { return abs2(sub2(a, b)); }

template <typename AccT, int MATH, bool RAINF>
struct QuadSweep {
    using SS = StepSums<float, AccT>;
    static constexpr int K = 4;

    static __device__ __forceinline__ void thresholds(QuadSeg &G, float wmax, float vseed)
    {
        const float thr = wmax > vseed ? wmax : vseed;
        G.thr = thr;
        G.thr2c = thr * thr * 0.999999f;
        const float t2 = thr * thr;
        G.T6 = thr >= 1e-6f ? t2 * t2 * t2 * 0.9998f : 0.0f;
    }

    // one iteration of the pipeline; J = (i - i0) & 3
    template <int J>
    static __device__ __forceinline__ void iter(QuadRing &R, QuadSeg &G, const PairK &c,
                                                const StepVals<float> &sv, const RunK<float> &rk,
                                                const StepK<float> *kp, SS &ss, int i)
    {
        constexpr int S1 = (J + 1) & 3;   // row i+1
        constexpr int S0 = J & 3;         // row i
        constexpr int Sm1 = (J + 3) & 3;  // row i-1
        constexpr int Sm2 = (J + 2) & 3;  // row i-2
        constexpr int Sm3 = (J + 1) & 3;  // row i-3
        constexpr int Sm4 = J & 3;        // row i-4
        const int pitch = G.pitch;
        const f2 z0 = bc2(0.0f);
        const f4 z04 = bc4(0.0f);

        // ---- loads: row i+1, and hmax / rain field of row i-1
        {
            const int off = G.o1;
            G.o1 += pitch;
            R.z[S1] = ld4(G.gz + off);
            R.h[S1] = ld4(G.hin + off);
            R.n[S1] = ld4(G.gn + off);
            const int offa = i + 1 + PF_ROWS <= G.nr + PADR - 1
                                 ? off + PF_ROWS * pitch
                                 : (G.nr + 2 * PADR - 1) * pitch + G.colo;
            prefetch_l2(G.gz + offa);
            prefetch_l2(G.hin + offa);
            prefetch_l2(G.gn + offa);
            const int off1 = off - 2 * pitch;
            R.hm[Sm1] = G.out_lane && i - 1 >= G.r0 && i - 1 < G.r1 ? ld4_rw(G.ghmax + off1) : z04;
            if constexpr (RAINF)
                R.cr[Sm1] = ld4(G.gcr + off1);
        }

        // ---- A: x faces of row i; y faces between rows i-1 and i
        {
            R.L[S0] = add4(R.z[S0], R.h[S0]);
            const f4 zr = right4(R.z[S0]), Lr = right4(R.L[S0]), nrr = right4(R.n[S0]);
            Face2 fx[2], fy[2];
#pragma unroll
            for (int q = 0; q < 2; q++) {
                fx[q] = face2_v<MATH>(R.L[S0].p[q], Lr.p[q], R.z[S0].p[q], zr.p[q], R.n[S0].p[q],
                                      nrr.p[q], c.dx, c.rdx, c);
                fy[q] = face2_v<MATH>(R.L[Sm1].p[q], R.L[S0].p[q], R.z[Sm1].p[q], R.z[S0].p[q],
                                      R.n[Sm1].p[q], R.n[S0].p[q], c.dx, c.rdx, c);
            }
            if constexpr (MATH == MATH_EXACT) {
                const bool crit = fx[0].cr0 || fx[0].cr1 || fx[1].cr0 || fx[1].cr1 || fy[0].cr0 ||
                                  fy[0].cr1 || fy[1].cr0 || fy[1].cr1;
                if (__any_sync(0xffffffffu, crit)) {
#pragma unroll
                    for (int q = 0; q < 2; q++) {
                        face2_crit(fx[q], c);
                        face2_crit(fy[q], c);
                    }
                }
            }
            f4 X, Y;
            bool cx[4], cy[4];
#pragma unroll
            for (int q = 0; q < 2; q++) {
                X.p[q] = face2_q<MATH>(fx[q], c.w, c, cx[2 * q], cx[2 * q + 1]);
                Y.p[q] = face2_q<MATH>(fy[q], c.w, c, cy[2 * q], cy[2 * q + 1]);
            }
            // faces are counted by the cell that holds them: x faces by row i,
            // y faces by row i-1; volume caps of the halves the exact
            // re-evaluation does not redo
            const bool ownA = G.out_lane && i >= G.r0 && i < G.r1;
            const bool ownB = G.out_lane && i - 1 >= G.r0 && i - 1 < G.r1;
#pragma unroll
            for (int q = 0; q < 2; q++) {
                if (ownA)
                    ss.capn += (unsigned)(cx[2 * q] && !fx[q].un0) +
                               (unsigned)(cx[2 * q + 1] && !fx[q].un1);
                if (ownB)
                    ss.capn += (unsigned)(cy[2 * q] && !fy[q].un0) +
                               (unsigned)(cy[2 * q + 1] && !fy[q].un1);
            }
            if constexpr (MATH == MATH_EXACT) {
                const bool any = fx[0].un0 || fx[0].un1 || fx[1].un0 || fx[1].un1 || fy[0].un0 ||
                                 fy[0].un1 || fy[1].un0 || fy[1].un1;
                if (__any_sync(0xffffffffu, any)) {
                    const f4 hr = right4(R.h[S0]);
#pragma unroll
                    for (int q = 0; q < 2; q++) {
                        if (fx[q].un0 || fx[q].un1) {
                            const Settled o =
                                face2_settle(X.p[q], fx[q].un0, fx[q].un1, R.z[S0].p[q],
                                             R.h[S0].p[q], R.n[S0].p[q], zr.p[q], hr.p[q],
                                             nrr.p[q], false, kp);
                            X.p[q] = o.Q;
                            if (ownA)
                                ss.capn += o.cap;
                        }
                        if (fy[q].un0 || fy[q].un1) {
                            const Settled o =
                                face2_settle(Y.p[q], fy[q].un0, fy[q].un1, R.z[Sm1].p[q],
                                             R.h[Sm1].p[q], R.n[Sm1].p[q], R.z[S0].p[q],
                                             R.h[S0].p[q], R.n[S0].p[q], false, kp);
                            Y.p[q] = o.Q;
                            if (ownB)
                                ss.capn += o.cap;
                        }
                    }
                }
            }
            R.X[S0] = X;
            R.Y[Sm1] = Y;
        }


        // ---- C: outflow volume and limiter of row i-1 (model.c:180-238,
        //      489-502), in the reference order +x, -x, +y, -y, open slots
        {
            const int r = i - 1;
            f4 out = sub4(max4(R.X[Sm1], z04), min4(left4(R.X[Sm1]), z04));
            out = add4(out, max4(R.Y[Sm1], z04));
            out = sub4(out, min4(R.Y[Sm2], z04));
            R.ko[Sm1] = 0u;
            R.qo[Sm1] = z04;
            if (G.edges) {
                const bool erow = (r == 0 && (G.edges & 1)) || (r == G.nr - 1 && (G.edges & 2));
                if (erow || G.edge_strip) {
                    const bool own = G.out_lane && r >= G.r0 && r < G.r1;
                    unsigned ko = 0u;
#pragma unroll
                    for (int q = 0; q < 2; q++) {
                        const OpenFaces o = open_faces2(
                            R.z[Sm1].p[q], R.h[Sm1].p[q], R.n[Sm1].p[q], r, G.cbase + 2 * q, G.nr,
                            G.nc, G.r_lo, G.r_hi, G.edges, own && ((G.colok >> (2 * q)) & 1u),
                            own && ((G.colok >> (2 * q + 1)) & 1u), kp);
                        ko |= o.ko << (8 * q);
                        R.qo[Sm1].p[q] = o.qo;
                        ss.capn += o.cap;
                        out.p[q] = add2(out.p[q], o.add);
                    }
                    R.ko[Sm1] = ko;
                }
            }
            f2 ov[2], hold[2];
            bool l[4];
#pragma unroll
            for (int q = 0; q < 2; q++) {
                ov[q] = mul2(out.p[q], c.dt);
                hold[q] = mul2(R.h[Sm1].p[q], c.A);
                const f2 hz = max2(hold[q], z0);
                l[2 * q] = lo2(ov[q]) > lo2(hz);
                l[2 * q + 1] = hi2(ov[q]) > hi2(hz);
            }
            R.s[Sm1] = bc4(1.0f);
            if (__any_sync(0xffffffffu, l[0] || l[1] || l[2] || l[3])) {
#pragma unroll
                for (int q = 0; q < 2; q++) {
                    const f2 o = sel2(l[2 * q], l[2 * q + 1], ov[q], bc2(1.0f));
                    f2 qv;
                    if constexpr (MATH == MATH_EXACT)
                        qv = div2_mk(hold[q], o, rcp2_nr(o));
                    else
                        qv = mul2(hold[q], rcp_2(o));
                    R.s[Sm1].p[q] = sel2(l[2 * q], l[2 * q + 1], qv, bc2(1.0f));
                }
            }
        }

        // ---- D: scaled discharges of the faces below and right of row i-2,
        //      net inflow, depth update, clamp, inflow, hmax/tmax, stage-E
        //      candidates (model.c:511-597)
        {
            const int r = i - 2;
            const bool row_out = r >= G.r0 && r < G.r1;
            const f4 s0 = R.s[Sm2];
            const f4 sr = right4(s0);
            f4 Qsx, Qsy;
#pragma unroll
            for (int q = 0; q < 2; q++) {
                Qsx.p[q] = fma2(min2(R.X[Sm2].p[q], z0), sr.p[q],
                                mul2(max2(R.X[Sm2].p[q], z0), s0.p[q]));
                Qsy.p[q] = fma2(min2(R.Y[Sm2].p[q], z0), R.s[Sm1].p[q],
                                mul2(max2(R.Y[Sm2].p[q], z0), s0.p[q]));
            }
            R.Qy[Sm2] = Qsy;
            f4 net = sub4(z04, Qsx);
            net = add4(net, left4(Qsx));
            net = sub4(net, Qsy);
            net = add4(net, R.Qy[Sm3]);
            bool cell[4];
#pragma unroll
            for (int j = 0; j < 4; j++)
                cell[j] = row_out && G.out_lane && ((G.colok >> j) & 1u);
            if (G.edges && __any_sync(0xffffffffu, R.ko[Sm2] != 0u)) {
                // open-edge outflow scaled by the cell's own limiter
                // (model.c:553-559), summed over its open slots
                float qb[4];
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const unsigned kk = (R.ko[Sm2] >> (4 * j)) & 15u;
                    qb[j] = open_sum<float>(get4(R.qo[Sm2], j) * get4(s0, j), __popc(kk));
                    if (cell[j] && kk)
                        ss.a_bnd += acc_mul<AccT, float>(sv.dt, qb[j]);
                }
                net.p[0] = sub2(net.p[0], mk2(qb[0], qb[1]));
                net.p[1] = sub2(net.p[1], mk2(qb[2], qb[3]));
            }
            f4 rain;
            rain.p[0] = rain.p[1] = c.rain;
            if constexpr (RAINF) {
                rain.p[0] = mul2_sep(R.cr[Sm2].p[0], bc2(sv.F));
                rain.p[1] = mul2_sep(R.cr[Sm2].p[1], bc2(sv.F));
            }
            f4 hu;
#pragma unroll
            for (int q = 0; q < 2; q++) {
                f2 dq;
                if constexpr (MATH == MATH_EXACT)
                    dq = div2_mk(net.p[q], c.A, c.invA);
                else
                    dq = mul2(net.p[q], c.invA);
                hu.p[q] = add2(R.h[Sm2].p[q], add2(mul2_sep(c.dt, dq), rain.p[q]));
            }
            {
                float u[4];
#pragma unroll
                for (int j = 0; j < 4; j++)
                    u[j] = get4(hu, j);
                if (__any_sync(0xffffffffu, u[0] < 0.0f || u[1] < 0.0f || u[2] < 0.0f ||
                                                u[3] < 0.0f)) {
#pragma unroll
                    for (int j = 0; j < 4; j++) {
                        if (u[j] < 0.0f) {
                            if (cell[j])
                                ss.a_clamp += acc_mul<AccT, float>(-u[j], sv.A);
                            u[j] = 0.0f;
                        }
                    }
                    hu.p[0] = mk2(u[0], u[1]);
                    hu.p[1] = mk2(u[2], u[3]);
                }
            }
            if (r == rk.inflow_r) {
                const int d = rk.inflow_c - G.cbase;
                if (d >= 0 && d < 4) {
                    f2 &pq = hu.p[d >> 1];
                    pq = (d & 1) ? mk2(lo2(pq), hi2(pq) + sv.inflow_dh)
                                 : mk2(lo2(pq) + sv.inflow_dh, hi2(pq));
                }
            }
            if constexpr (sizeof(AccT) == 4) {
#pragma unroll
                for (int j = 0; j < 4; j++)
                    if (cell[j])
                        ss.a_rain += sv.A * get4(rain, j);
            } else if constexpr (RAINF) {
                double rs = 0.0;
#pragma unroll
                for (int j = 0; j < 4; j++)
                    rs += cell[j] ? (double)get4(rain, j) : 0.0;
                ss.rain_sum += rs;
            }
            // new level for stage E (NaN outside the grid: no neighbour
            // there); cells outside the grid keep their padding depth
            f4 Ln = add4(R.z[Sm2], hu);
            f4 hkeep = hu;
            if (G.edge_strip || r < G.r_lo || r >= G.r_hi) {
                const bool rin = r >= G.r_lo && r < G.r_hi;
#pragma unroll
                for (int q = 0; q < 2; q++) {
                    const bool in0 = rin && ((G.colok >> (2 * q)) & 1u);
                    const bool in1 = rin && ((G.colok >> (2 * q + 1)) & 1u);
                    Ln.p[q] = sel2(in0, in1, Ln.p[q], bc2(__int_as_float(0x7fc00000)));
                    hkeep.p[q] = sel2(in0, in1, hu.p[q], R.h[Sm2].p[q]);
                }
            }
            R.Ln[Sm2] = Ln;
            R.hn[Sm2] = hu;
            // stage-E candidates: wet output cells whose critical velocity
            // sqrt(g h) may exceed the warp's threshold (margin 1e-6)
            unsigned ef = 0u;
            if (sv.want_v) {
                const bool t = G.thr > 0.0f;
#pragma unroll
                for (int q = 0; q < 2; q++) {
                    const f2 gh = mul2(c.g, hu.p[q]);
                    if (cell[2 * q] && lo2(hu.p[q]) >= c.tau_h && !(t && lo2(gh) <= G.thr2c))
                        ef |= 1u << (2 * q);
                    if (cell[2 * q + 1] && hi2(hu.p[q]) >= c.tau_h && !(t && hi2(gh) <= G.thr2c))
                        ef |= 2u << (2 * q);
                }
            }
#pragma unroll
            for (int q = 0; q < 2; q++) {
                const f2 n2 = mul2(R.n[Sm2].p[q], R.n[Sm2].p[q]);
                R.n6[Sm2].p[q] = mul2(mul2(n2, n2), n2);
            }
            R.ef[Sm2] = ef;
            // hmax / tmax of output cells
            const f4 hmo = R.hm[Sm2];
            bool rise[4];
#pragma unroll
            for (int j = 0; j < 4; j++)
                rise[j] = cell[j] && get4(hu, j) > get4(hmo, j);
            if (row_out && G.out_lane) {
                // hmax written back whether or not it rose, tmax where it rose
                const int off2 = G.o1 - 4 * pitch;              // row i-2
                st4(G.hout + off2, hkeep);
                f4 hmn;
                hmn.p[0] = sel2(rise[0], rise[1], hu.p[0], hmo.p[0]);
                hmn.p[1] = sel2(rise[2], rise[3], hu.p[1], hmo.p[1]);
                st4(G.ghmax + off2, hmn);
#pragma unroll
                for (int j = 0; j < 4; j++)
                    if (rise[j])
                        G.gtmax[off2 + j] = sv.tmax_val;
            }
        }

        // ---- E: next step's stable velocity of row i-3 from the new levels
        //      of rows i-4..i-2 (physics.h:158-217), for the candidates
        if (sv.want_v && __any_sync(0xffffffffu, R.ef[Sm3] != 0u)) {
            const int r = i - 3;
            const f4 la = R.Ln[Sm3];
            const f4 lr = right4(la), ll = left4(la);
            f4 mo;
#pragma unroll
            for (int q = 0; q < 2; q++) {
                f2 m = max2(abs2d(la.p[q], lr.p[q]), abs2d(la.p[q], ll.p[q]));
                m = max2(m, max2(abs2d(la.p[q], R.Ln[Sm2].p[q]), abs2d(la.p[q], R.Ln[Sm4].p[q])));
                mo.p[q] = max2(m, z0);
            }
            if (G.edges) {
                const bool erow = (r == 0 && (G.edges & 1)) || (r == G.nr - 1 && (G.edges & 2));
                if (erow || G.edge_strip) {
                    // the open virtual neighbour z - S_bnd*dx, h = 0 (physics.h:183-189)
                    const int off3 = G.o1 - 5 * pitch;          // row i-3
                    const f4 z3 = ld4(G.gz + off3);
#pragma unroll
                    for (int q = 0; q < 2; q++) {
                        const f2 dv = abs2(sub2(la.p[q], sub2(z3.p[q], bc2(sv.k.S_bnd * sv.k.dx))));
#pragma unroll
                        for (int h = 0; h < 2; h++) {
                            const int cc = G.cbase + 2 * q + h;
                            if (erow || (cc == 0 && (G.edges & 4)) ||
                                (cc == G.nc - 1 && (G.edges & 8)))
                                put2(mo.p[q], h, fmaxf(get2(mo.p[q], h), get2(dv, h)));
                        }
                    }
                }
            }
            // bound: v^6 <= h^4 S^3 / n^6 (S = the largest slope), against thr^6
            const unsigned ef = R.ef[Sm3];
            bool x[4];
#pragma unroll
            for (int q = 0; q < 2; q++) {
                const f2 S = mul2(mo.p[q], c.rdx);
                const f2 hv = R.hn[Sm3].p[q];
                const f2 h2 = mul2(hv, hv);
                const f2 lhs = mul2(mul2(h2, h2), mul2(mul2(S, S), S));
                const f2 rhs = mul2(R.n6[Sm3].p[q], bc2(G.T6));
                x[2 * q] = ((ef >> (2 * q)) & 1u) && (lo2(lhs) >= lo2(rhs) || lo2(lhs) < 1e-30f);
                x[2 * q + 1] =
                    ((ef >> (2 * q + 1)) & 1u) && (hi2(lhs) >= hi2(rhs) || hi2(lhs) < 1e-30f);
            }
            if (__any_sync(0xffffffffu, x[0] || x[1] || x[2] || x[3])) {
                const int off3 = G.o1 - 5 * pitch;              // row i-3
                const f4 n3 = ld4(G.gn + off3);
                float vm = ss.vmax;
#pragma unroll
                for (int q = 0; q < 2; q++)
                    if (x[2 * q] || x[2 * q + 1])
                        vm = pair_velocity<4, MATH>(vm, x[2 * q], x[2 * q + 1], mo.p[q], z0,
                                                    R.hn[Sm3].p[q], n3.p[q], kp);
                ss.vmax = vm;
                thresholds(G, warp_max_nonneg(vm), sv.vseed);
            }
        }
    }

    // One warp streams output rows [r0, r1) of one 128-column strip.
    static __device__ __forceinline__ void run(const GridD<float> &g, const RunK<float> &rk,
                                               const StepVals<float> &sv, const StepK<float> *kp,
                                               int strip, int r0, int r1, int lane, SS &ss)
    {
        using Gm = Geom<4>;
        QuadSeg G;
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
        G.cbase = strip * Gm::OW - Gm::HL + lane * 4;
        G.colo = G.cbase + PADC;
        G.out_lane = lane * 4 >= Gm::HL && lane * 4 < Gm::HL + Gm::OW;
        G.colok = 0u;
#pragma unroll
        for (int j = 0; j < 4; j++)
            G.colok |= (G.cbase + j >= 0 && G.cbase + j < g.nc) ? 1u << j : 0u;
        G.edges = rk.open ? (rk.edge_n ? 1 : 0) | (rk.edge_s ? 2 : 0) | (rk.edge_w ? 4 : 0) |
                                (rk.edge_e ? 8 : 0)
                          : 0;
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

        // iterations i0 .. r1+2; the extra leading iterations compute rows
        // above the segment's halo only
        const int n_it = ((r1 - r0 + 6) + 3) & ~3;
        const int i0 = r1 + 3 - n_it;

        QuadRing R;
        const f4 z04 = bc4(0.0f);
#pragma unroll
        for (int q = 0; q < 4; q++) {
            R.z[q] = R.h[q] = R.n[q] = R.L[q] = z04;
            R.X[q] = R.Y[q] = z04;
            R.s[q] = bc4(1.0f);
            R.Qy[q] = R.hn[q] = R.n6[q] = R.hm[q] = R.cr[q] = R.qo[q] = z04;
            R.Ln[q] = bc4(__int_as_float(0x7fc00000));
            R.ko[q] = R.ef[q] = 0u;
        }
        {
            const int off = (i0 + PADR) * G.pitch + G.colo;
            R.z[0] = ld4(G.gz + off);
            R.h[0] = ld4(G.hin + off);
            R.n[0] = ld4(G.gn + off);
        }
        G.o1 = (i0 + 1 + PADR) * G.pitch + G.colo;
        for (int i = i0; i < i0 + n_it; i++) {
            iter<0>(R, G, c, sv, rk, kp, ss, i);
            rotate_quad(R);
        }
        // uniform rain on LAND output cells, counted per lane
        if constexpr (sizeof(AccT) == 8 && !RAINF) {
            if (G.out_lane)
                ss.rain_cells += (long long)(r1 - r0) * __popc(G.colok);
        }
    }
};
}  // namespace fcab
