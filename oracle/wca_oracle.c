/*
 * CPU oracle for the FloodCA WCA flood step -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference algorithm, written for this project.
 * Each function names the reference lines it follows (paths relative to the
 * FloodCA source tree). It is the checker for the CUDA path: only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg may call it.
 *
 * Compile with -ffp-contract=off (see oracle/Makefile) so that every float
 * operation rounds once, like the reference parity build.
 */
#include "wca_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define DAY_S 86400.0

int or_real_size(void) { return (int)sizeof(oreal); }

/* Physical constants in reference precision (FloodCA src/common/config.c:8-45
 * stores them as `real`). */
typedef struct Phys {
    oreal dx, A, g, alpha, tau_h, tau_l, z_sea, dt_max, dt_min, S_bnd;
    int U, K, open;
} Phys;

static void phys_from(const OrParams *p, Phys *q)
{
    q->dx = (oreal)p->dx;
    q->A = q->dx * q->dx;
    q->g = (oreal)p->g;
    q->alpha = (oreal)p->alpha;
    q->tau_h = (oreal)p->tau_h;
    q->tau_l = (oreal)p->tau_l;
    q->z_sea = (oreal)p->z_sea;
    q->dt_max = (oreal)p->dt_max;
    q->dt_min = (oreal)p->dt_min;
    q->S_bnd = (oreal)p->S_bnd;
    q->U = p->U > 0 ? p->U : 1;
    q->K = p->K;
    q->open = p->boundary == 0;
}

/* hf^(2/3) via a double cube root of hf*hf (physics.h:19-24). */
oreal or_cbrt_sq(oreal hf)
{
    double sq = (double)hf * (double)hf;
    return (oreal)cbrt(sq);
}

/* A face exists unless either side is WALL or both are SEA (physics.h:26-35). */
static int face_exists(uint8_t ma, uint8_t mb)
{
    if (ma == OR_WALL || mb == OR_WALL)
        return 0;
    return !(ma == OR_SEA && mb == OR_SEA);
}

/* Face width: dx for K=4, (sqrt2-1)dx for K=8 (physics.h:37-43). */
static oreal orth_width(oreal dx, int K)
{
    return K == 8 ? ((oreal)sqrt(2.0) - (oreal)1) * dx : dx;
}

/* Centre distance of a diagonal face (physics.h:45-48). */
static oreal diag_dist(oreal dx) { return (oreal)sqrt(2.0) * dx; }

/* Signed discharge a->b: Manning velocity, critical-depth cap, then a volume
 * cap against the level difference (physics.h:51-125). */
static oreal face_flux(oreal za, oreal ha, oreal na, uint8_t ma, oreal zb, oreal hb, oreal nb,
                       uint8_t mb, oreal d, oreal w, oreal dt, int K, oreal A, const Phys *q,
                       int *cap)
{
    oreal zea, zeb, la, lb, dL, adL, hf, nf, S, v, vcr, Qm, Qc;
    *cap = 0;
    if (ma == OR_WALL || mb == OR_WALL)
        return 0;
    zea = ma == OR_SEA ? q->z_sea : za;
    zeb = mb == OR_SEA ? q->z_sea : zb;
    la = zea + (ma == OR_SEA ? (oreal)0 : ha);
    lb = zeb + (mb == OR_SEA ? (oreal)0 : hb);
    dL = la - lb;
    adL = dL < 0 ? -dL : dL;
    if (adL < q->tau_l)
        return 0;
    hf = (la > lb ? la : lb) - (zea > zeb ? zea : zeb);
    if (hf < q->tau_h)
        return 0;
    if ((dL > 0 ? ma : mb) == OR_SEA)
        return 0;
    if (ma == OR_SEA)
        nf = nb;
    else if (mb == OR_SEA)
        nf = na;
    else
        nf = (oreal)0.5 * (na + nb);
    if (nf < (oreal)1e-12)
        nf = (oreal)1e-12;
    S = adL / d;
    v = ((oreal)1 / nf) * or_cbrt_sq(hf) * (oreal)sqrt((double)S);
    vcr = (oreal)sqrt((double)q->g * (double)hf);
    if (v > vcr)
        v = vcr;
    Qm = v * hf * w;
    if (dt > 0 && K > 0) {
        Qc = adL * A / ((oreal)(2 * K) * dt);
        if (Qc < Qm) {
            *cap = 1;
            Qm = Qc;
        }
    }
    return dL > 0 ? Qm : -Qm;
}

oreal or_face_flux(oreal za, oreal ha, oreal na, uint8_t ma, oreal zb, oreal hb, oreal nb,
                   uint8_t mb, oreal d, oreal w, oreal dt, int K, oreal A, const OrParams *p,
                   int *cap)
{
    Phys q;
    phys_from(p, &q);
    return face_flux(za, ha, na, ma, zb, hb, nb, mb, d, w, dt, K, A, &q, cap);
}

/* Outflow limiter s = held volume / outflow volume when it would overdraw
 * (physics.h:127-134). */
static oreal limiter(oreal out_vol, oreal h, oreal A)
{
    oreal hold = h * A;
    if (out_vol > hold && out_vol > 0)
        return hold / out_vol;
    return 1;
}

/* Water-surface level of a cell as seen from a neighbour (physics.h:136-145). */
static oreal level_of(uint8_t m, oreal z, oreal h, const Phys *q)
{
    if (m == OR_SEA)
        return q->z_sea;
    if (m == OR_WALL)
        return z;
    return z + h;
}

/* Largest |slope| to an existing neighbour, plus the open-edge virtual
 * neighbour (physics.h:158-191). */
static oreal cell_smax(const oreal *z, const oreal *h, const uint8_t *mask, int r, int c, int nr,
                       int nc, const Phys *q, int open_edge)
{
    long a = (long)r * nc + c;
    uint8_t ma = mask[a];
    oreal la = z[a] + h[a], Smax = 0, S;
    oreal dd = diag_dist(q->dx);
    struct { int ok; long b; oreal d; } nb[8] = {
        {c + 1 < nc, a + 1, q->dx},
        {c - 1 >= 0, a - 1, q->dx},
        {r + 1 < nr, a + nc, q->dx},
        {r - 1 >= 0, a - nc, q->dx},
        {r + 1 < nr && c + 1 < nc, a + nc + 1, dd},
        {r + 1 < nr && c - 1 >= 0, a + nc - 1, dd},
        {r - 1 >= 0 && c + 1 < nc, a - nc + 1, dd},
        {r - 1 >= 0 && c - 1 >= 0, a - nc - 1, dd},
    };
    int k, kn = q->K == 8 ? 8 : 4;
    for (k = 0; k < kn; k++) {
        oreal dL;
        if (!nb[k].ok || !face_exists(ma, mask[nb[k].b]))
            continue;
        dL = la - level_of(mask[nb[k].b], z[nb[k].b], h[nb[k].b], q);
        S = (dL < 0 ? -dL : dL) / nb[k].d;
        if (S > Smax)
            Smax = S;
    }
    if (open_edge) {
        oreal lv = z[a] - q->S_bnd * q->dx, dL = la - lv;
        S = (dL < 0 ? -dL : dL) / q->dx;
        if (S > Smax)
            Smax = S;
    }
    return Smax;
}

/* Per-cell stable step alpha*dx/v (physics.h:193-217). */
static oreal cell_dt(oreal h, oreal n, oreal Smax, const Phys *q)
{
    oreal v, vcr;
    if (h < q->tau_h)
        return q->dt_max;
    if (n < (oreal)1e-12)
        n = (oreal)1e-12;
    if (Smax < 0)
        Smax = 0;
    v = ((oreal)1 / n) * or_cbrt_sq(h) * (oreal)sqrt((double)Smax);
    vcr = (oreal)sqrt((double)q->g * (double)h);
    if (v > vcr)
        v = vcr;
    if (v < (oreal)1e-6)
        v = (oreal)1e-6;
    return q->alpha * q->dx / v;
}

static int edge_open(const OrParams *p, const Phys *q, int r, int c, int nr, int nc)
{
    return q->open && ((c == 0 && p->edge_w) || (c == nc - 1 && p->edge_e) ||
                       (r == 0 && p->edge_n) || (r == nr - 1 && p->edge_s));
}

/* Global stable step: min over wet LAND cells, clamped to [dt_min, dt_max]
 * (FloodCA src/common/model.c:111-156). */
static oreal compute_dt(int nr, int nc, const oreal *z, const oreal *h, const oreal *n,
                        const uint8_t *mask, const OrParams *p, const Phys *q, OrAcc *acc)
{
    oreal dtmin = q->dt_max;
    int r, any = 0;
#pragma omp parallel for schedule(static) reduction(min : dtmin) reduction(+ : any)
    for (r = 0; r < nr; r++) {
        int c;
        for (c = 0; c < nc; c++) {
            long a = (long)r * nc + c;
            oreal dta;
            if (mask[a] != OR_LAND || h[a] < q->tau_h)
                continue;
            any++;
            dta = cell_dt(h[a], n[a],
                          cell_smax(z, h, mask, r, c, nr, nc, q, edge_open(p, q, r, c, nr, nc)),
                          q);
            if (dta < dtmin)
                dtmin = dta;
        }
    }
    if (!any)
        dtmin = q->dt_max;
    if (dtmin < q->dt_min) {
        dtmin = q->dt_min;
        acc->dt_min_hits++;
    }
    if (dtmin > q->dt_max)
        dtmin = q->dt_max;
    return dtmin;
}

/* Unit hyetograph integral over [t, t+dt]: uniform 1/86400 or a triangle of
 * base D_h hours peaking at phi*D_h (FloodCA src/common/rain.c:8-67). */
static double tri_f(double t, double T, double tp)
{
    if (t < 0.0 || t >= T || T <= 0.0)
        return 0.0;
    if (t < tp)
        return tp <= 0.0 ? 0.0 : (2.0 / T) * (t / tp);
    return T - tp <= 0.0 ? 0.0 : (2.0 / T) * ((T - t) / (T - tp));
}

double or_hyeto_integral(const OrParams *p, double t, double dt)
{
    double t1, T, tp, sum = 0.0, a;
    if (dt <= 0.0)
        return 0.0;
    t1 = t + dt;
    if (p->hyeto == 1)
        return dt / DAY_S;
    T = (double)(oreal)p->D_h * 3600.0;
    tp = (double)(oreal)p->phi * T;
    if (t1 <= 0.0 || t >= T)
        return 0.0;
    if (t < 0.0)
        t = 0.0;
    if (t1 > T)
        t1 = T;
    a = t;
    while (a < t1 - 1e-15) {
        double b = (a < tp && t1 > tp) ? tp : t1;
        sum += 0.5 * (tri_f(a, T, tp) + tri_f(b, T, tp)) * (b - a);
        a = b;
    }
    return sum;
}

/* Next step event: T_sim, next day boundary, next out_every multiple
 * (FloodCA src/common/rain.c:69-93), plus the rain_end extension. */
double or_next_event_time(const OrParams *p, double t)
{
    double t_next = (double)(oreal)p->T_sim, t_day, oe;
    t_day = (floor(t / DAY_S) + 1.0) * DAY_S;
    if (t_day - t < 1e-9)
        t_day += DAY_S;
    if (t_day < t_next)
        t_next = t_day;
    oe = (double)(oreal)p->out_every;
    if (oe > 0.0) {
        double t_out = (floor(t / oe) + 1.0) * oe;
        if (t_out - t < 1e-9)
            t_out += oe;
        if (t_out < t_next)
            t_next = t_out;
    }
    if (p->rain_end > 0.0 && p->rain_end - t >= 1e-9 && p->rain_end < t_next)
        t_next = p->rain_end;
    return t_next;
}

/* Exact integral of the triangular inflow hydrograph over [t, t+dt]. */
static double inflow_q(const OrParams *p, double t)
{
    double tp = p->inflow_t_peak, te = p->inflow_t_end;
    if (t <= 0.0 || t >= te)
        return 0.0;
    if (t <= tp)
        return tp > 0.0 ? p->inflow_peak * (t / tp) : p->inflow_peak;
    return te > tp ? p->inflow_peak * ((te - t) / (te - tp)) : 0.0;
}

double or_inflow_volume(const OrParams *p, double t, double dt)
{
    double t1 = t + dt, a, sum = 0.0;
    if (p->inflow_cell < 0 || dt <= 0.0)
        return 0.0;
    if (t < 0.0)
        t = 0.0;
    if (t1 > p->inflow_t_end)
        t1 = p->inflow_t_end;
    a = t;
    while (a < t1) {
        double b = (a < p->inflow_t_peak && t1 > p->inflow_t_peak) ? p->inflow_t_peak : t1;
        sum += 0.5 * (inflow_q(p, a) + inflow_q(p, b)) * (b - a);
        a = b;
    }
    return sum;
}

double or_volume_land(int nr, int nc, const oreal *h, const uint8_t *mask, double dx)
{
    oreal A = (oreal)dx * (oreal)dx;
    double V = 0.0;
    long i, N = (long)nr * nc;
#pragma omp parallel for schedule(static) reduction(+ : V)
    for (i = 0; i < N; i++)
        if (mask[i] == OR_LAND)
            V += (double)h[i] * (double)A;
    return V;
}

void or_acc_init(OrAcc *acc, int nr, int nc, const oreal *h, const uint8_t *mask, double dx)
{
    memset(acc, 0, sizeof(*acc));
    acc->V0 = or_volume_land(nr, nc, h, mask, dx);
    acc->V = acc->V0;
    acc->force_day = -1;
}

double or_mass_error(const OrAcc *acc)
{
    double den = acc->V_rain + acc->V_in + acc->V0;
    if (den < 1e-30)
        den = 1e-30;
    return fabs(acc->V + acc->V_sea + acc->V_bnd - acc->V_rain - acc->V_in - acc->V0 -
                acc->clamp_err) /
           den;
}

typedef struct Work {
    oreal *Qx, *Qy, *Qd1, *Qd2, *Qop, *s;
} Work;

/* Sum of positive outgoing face discharge, in the reference face order
 * +x, -x, +y, -y, [d1+, d1-, d2+, d2-], then the four open slots
 * (FloodCA src/common/model.c:180-238). */
static oreal outflow_sum(const Work *w, int r, int c, int nr, int nc, int K)
{
    long a = (long)r * nc + c;
    oreal out = 0, Q;
    if (c + 1 < nc && (Q = w->Qx[(long)r * (nc - 1) + c]) > 0)
        out += Q;
    if (c > 0 && (Q = w->Qx[(long)r * (nc - 1) + c - 1]) < 0)
        out += -Q;
    if (r + 1 < nr && (Q = w->Qy[(long)r * nc + c]) > 0)
        out += Q;
    if (r > 0 && (Q = w->Qy[(long)(r - 1) * nc + c]) < 0)
        out += -Q;
    if (K == 8) {
        if (r + 1 < nr && c + 1 < nc && (Q = w->Qd1[(long)r * (nc - 1) + c]) > 0)
            out += Q;
        if (r > 0 && c > 0 && (Q = w->Qd1[(long)(r - 1) * (nc - 1) + c - 1]) < 0)
            out += -Q;
        if (r + 1 < nr && c > 0 && (Q = w->Qd2[(long)r * (nc - 1) + c - 1]) > 0)
            out += Q;
        if (r > 0 && c + 1 < nc && (Q = w->Qd2[(long)(r - 1) * (nc - 1) + c]) < 0)
            out += -Q;
    }
    out += w->Qop[4 * a] + w->Qop[4 * a + 1] + w->Qop[4 * a + 2] + w->Qop[4 * a + 3];
    return out;
}

/* Net inflow of cell (r,c) from limiter-scaled discharges, adding LAND->SEA
 * outflow volume to *sea (FloodCA src/common/model.c:241-319). */
static oreal net_inflow(const Work *w, const uint8_t *mask, int r, int c, int nr, int nc, int K,
                        oreal dt, double *sea)
{
    long a = (long)r * nc + c;
    int land = mask[a] == OR_LAND;
    oreal net = 0, Q, Qo;
#define SEA_OUT(bidx, cond)                                                                  \
    if (land && mask[bidx] == OR_SEA && (cond))                                              \
        *sea += (double)dt * (double)((Q) < 0 ? -(Q) : (Q));
    if (c + 1 < nc) {
        Q = w->Qx[(long)r * (nc - 1) + c];
        net -= Q;
        SEA_OUT(a + 1, Q > 0)
    }
    if (c > 0) {
        Q = w->Qx[(long)r * (nc - 1) + c - 1];
        net += Q;
        SEA_OUT(a - 1, Q < 0)
    }
    if (r + 1 < nr) {
        Q = w->Qy[(long)r * nc + c];
        net -= Q;
        SEA_OUT(a + nc, Q > 0)
    }
    if (r > 0) {
        Q = w->Qy[(long)(r - 1) * nc + c];
        net += Q;
        SEA_OUT(a - nc, Q < 0)
    }
    if (K == 8) {
        if (r + 1 < nr && c + 1 < nc) {
            Q = w->Qd1[(long)r * (nc - 1) + c];
            net -= Q;
            SEA_OUT(a + nc + 1, Q > 0)
        }
        if (r > 0 && c > 0) {
            Q = w->Qd1[(long)(r - 1) * (nc - 1) + c - 1];
            net += Q;
            SEA_OUT(a - nc - 1, Q < 0)
        }
        if (r + 1 < nr && c > 0) {
            Q = w->Qd2[(long)r * (nc - 1) + c - 1];
            net -= Q;
            SEA_OUT(a + nc - 1, Q > 0)
        }
        if (r > 0 && c + 1 < nc) {
            Q = w->Qd2[(long)(r - 1) * (nc - 1) + c];
            net += Q;
            SEA_OUT(a - nc + 1, Q < 0)
        }
    }
#undef SEA_OUT
    Qo = w->Qop[4 * a] + w->Qop[4 * a + 1] + w->Qop[4 * a + 2] + w->Qop[4 * a + 3];
    net -= Qo;
    return net;
}

/* Open-edge discharge to a virtual neighbour at z - S_bnd*dx with h = 0,
 * clipped at zero (FloodCA src/common/model.c:166-177). */
static oreal open_flux(oreal z, oreal h, oreal n, uint8_t m, const Phys *q, oreal dt, int *cap)
{
    oreal Q = face_flux(z, h, n, m, z - q->S_bnd * q->dx, 0, n, OR_LAND, q->dx,
                        orth_width(q->dx, q->K), dt, q->K, q->A, q, cap);
    return Q < 0 ? 0 : Q;
}

/* One step (FloodCA src/common/model.c:321-605). Returns 1 if a step was
 * taken, 0 if dt was not positive, -1 on a forcing error. */
static int step_once(int nr, int nc, const oreal *z, oreal *h, const oreal *n, const oreal *C,
                     oreal *Rday, const uint8_t *mask, oreal *hmax, oreal *tmax,
                     const OrParams *p, const Phys *q, OrAcc *acc, Work *w,
                     const oreal *force_rday)
{
    long N = (long)nr * nc, i;
    int r, K = q->K, hit = 0;
    oreal dx = q->dx, A = q->A, wd = orth_width(dx, K), dd = diag_dist(dx), dt;
    double t_next, remain, F;
    long long capa = 0, capt = 0;
    double v_rain = 0, clamp = 0, v_sea = 0, v_bnd = 0, V_in = 0;
    long inflow = p->inflow_cell;

    if (p->n_force_days > 0 && force_rday) {
        int d = acc->t < 0.0 ? 0 : (int)floor(acc->t / DAY_S);
        if (d >= p->n_force_days)
            d = p->n_force_days - 1;
        if (d != acc->force_day) {
            oreal lam = (oreal)p->lambda;
            memcpy(Rday, force_rday + (long)d * N, (size_t)N * sizeof(oreal));
            if (lam != (oreal)1)
                for (i = 0; i < N; i++)
                    Rday[i] *= lam;
            acc->force_day = d;
        }
    }
    if (acc->step % q->U == 0)
        acc->dt_base = (double)compute_dt(nr, nc, z, h, n, mask, p, q, acc);
    dt = (oreal)acc->dt_base;
    t_next = or_next_event_time(p, acc->t);
    remain = t_next - acc->t;
    if (remain <= (double)dt) {
        if (remain < 0)
            remain = 0;
        dt = (oreal)remain;
        hit = 1;
    }
    if (dt <= 0)
        return 0;
    F = (p->rain_end <= 0.0 || p->rain_end - acc->t >= 1e-9)
            ? or_hyeto_integral(p, acc->t, (double)dt)
            : 0.0;

#pragma omp parallel for schedule(static) reduction(+ : capa, capt)
    for (r = 0; r < nr; r++) {
        int c, cap;
        for (c = 0; c < nc; c++) {
            long a = (long)r * nc + c;
            if (c + 1 < nc) {
                w->Qx[(long)r * (nc - 1) + c] = face_flux(z[a], h[a], n[a], mask[a], z[a + 1],
                                                          h[a + 1], n[a + 1], mask[a + 1], dx,
                                                          wd, dt, K, A, q, &cap);
                capa += cap;
                capt++;
            }
            if (r + 1 < nr) {
                w->Qy[(long)r * nc + c] = face_flux(z[a], h[a], n[a], mask[a], z[a + nc],
                                                    h[a + nc], n[a + nc], mask[a + nc], dx, wd,
                                                    dt, K, A, q, &cap);
                capa += cap;
                capt++;
            }
            if (K == 8 && r + 1 < nr && c + 1 < nc) {
                long b1 = a + nc + 1, a2 = a + 1, b2 = a + nc;
                w->Qd1[(long)r * (nc - 1) + c] =
                    face_flux(z[a], h[a], n[a], mask[a], z[b1], h[b1], n[b1], mask[b1], dd, wd,
                              dt, K, A, q, &cap);
                capa += cap;
                capt++;
                w->Qd2[(long)r * (nc - 1) + c] =
                    face_flux(z[a2], h[a2], n[a2], mask[a2], z[b2], h[b2], n[b2], mask[b2], dd,
                              wd, dt, K, A, q, &cap);
                capa += cap;
                capt++;
            }
            if (q->open && mask[a] == OR_LAND) {
                int side[4] = {c == 0 && p->edge_w, c == nc - 1 && p->edge_e,
                               r == 0 && p->edge_n, r == nr - 1 && p->edge_s};
                int k;
                for (k = 0; k < 4; k++) {
                    if (!side[k])
                        continue;
                    w->Qop[4 * a + k] = open_flux(z[a], h[a], n[a], mask[a], q, dt, &cap);
                    capa += cap;
                    capt++;
                }
            }
        }
    }
    acc->cap_active += capa;
    acc->cap_total += capt;

#pragma omp parallel for schedule(static)
    for (r = 0; r < nr; r++) {
        int c;
        for (c = 0; c < nc; c++) {
            long a = (long)r * nc + c;
            oreal ov = outflow_sum(w, r, c, nr, nc, K) * dt;
            w->s[a] = mask[a] == OR_LAND ? limiter(ov, h[a], A) : (oreal)1;
        }
    }

    /* Scale every face by its upwind cell's limiter (model.c:511-559). */
#pragma omp parallel for schedule(static)
    for (r = 0; r < nr; r++) {
        int c;
        for (c = 0; c < nc; c++) {
            long a = (long)r * nc + c;
            oreal Q;
            if (c + 1 < nc) {
                Q = w->Qx[(long)r * (nc - 1) + c];
                w->Qx[(long)r * (nc - 1) + c] = Q * (Q >= 0 ? w->s[a] : w->s[a + 1]);
            }
            if (r + 1 < nr) {
                Q = w->Qy[(long)r * nc + c];
                w->Qy[(long)r * nc + c] = Q * (Q >= 0 ? w->s[a] : w->s[a + nc]);
            }
            if (K == 8 && r + 1 < nr && c + 1 < nc) {
                Q = w->Qd1[(long)r * (nc - 1) + c];
                w->Qd1[(long)r * (nc - 1) + c] = Q * (Q >= 0 ? w->s[a] : w->s[a + nc + 1]);
                Q = w->Qd2[(long)r * (nc - 1) + c];
                w->Qd2[(long)r * (nc - 1) + c] = Q * (Q >= 0 ? w->s[a + 1] : w->s[a + nc]);
            }
            w->Qop[4 * a] *= w->s[a];
            w->Qop[4 * a + 1] *= w->s[a];
            w->Qop[4 * a + 2] *= w->s[a];
            w->Qop[4 * a + 3] *= w->s[a];
        }
    }

    if (inflow >= 0 && inflow < N && mask[inflow] == OR_LAND)
        V_in = or_inflow_volume(p, acc->t, (double)dt);

#pragma omp parallel for schedule(static) reduction(+ : v_rain, clamp, v_sea, v_bnd)
    for (r = 0; r < nr; r++) {
        int c;
        for (c = 0; c < nc; c++) {
            long a = (long)r * nc + c;
            double sea = 0;
            oreal net = net_inflow(w, mask, r, c, nr, nc, K, dt, &sea), Qo, rain, ha;
            v_sea += sea;
            Qo = w->Qop[4 * a] + w->Qop[4 * a + 1] + w->Qop[4 * a + 2] + w->Qop[4 * a + 3];
            v_bnd += (double)dt * (double)Qo;
            if (mask[a] != OR_LAND)
                continue;
            rain = C[a] * Rday[a] * (oreal)F;
            v_rain += (double)A * (double)rain;
            ha = h[a] + (dt * (net / A) + rain);
            if (ha < 0) {
                clamp += (double)(-ha) * (double)A;
                ha = 0;
            }
            if (a == inflow)
                ha = ha + (oreal)(V_in / (double)A);
            h[a] = ha;
            if (ha > hmax[a]) {
                hmax[a] = ha;
                tmax[a] = (oreal)(acc->t + (double)dt);
            }
        }
    }
    acc->V_rain += v_rain;
    acc->clamp_err += clamp;
    acc->V_sea += v_sea;
    acc->V_bnd += v_bnd;
    acc->V_in += V_in;
    acc->t = hit ? t_next : acc->t + (double)dt;
    acc->step++;
    return 1;
}

int or_run(int nr, int nc, const oreal *z, oreal *h, const oreal *n, const oreal *C, oreal *Rday,
           const uint8_t *mask, oreal *hmax, oreal *tmax, const OrParams *p, OrAcc *acc,
           int max_calls, const oreal *force_rday)
{
    Phys q;
    Work w;
    long N = (long)nr * nc;
    long nq = N > 0 ? N : 1;
    int max_steps = p->steps > 0 ? p->steps : 2000000000, taken = 0;

    phys_from(p, &q);
    memset(&w, 0, sizeof(w));
    w.Qx = (oreal *)calloc((size_t)nq, sizeof(oreal));
    w.Qy = (oreal *)calloc((size_t)nq, sizeof(oreal));
    w.Qd1 = (oreal *)calloc((size_t)nq, sizeof(oreal));
    w.Qd2 = (oreal *)calloc((size_t)nq, sizeof(oreal));
    w.Qop = (oreal *)calloc((size_t)(4 * nq), sizeof(oreal));
    w.s = (oreal *)calloc((size_t)nq, sizeof(oreal));
    if (!w.Qx || !w.Qy || !w.Qd1 || !w.Qd2 || !w.Qop || !w.s) {
        taken = -1;
        goto out;
    }
    while (acc->step < max_steps && taken < max_calls) {
        double t_before = acc->t;
        int rc;
        if (p->steps <= 0 && acc->t >= (double)(oreal)p->T_sim - 1e-15)
            break;
        rc = step_once(nr, nc, z, h, n, C, Rday, mask, hmax, tmax, p, &q, acc, &w, force_rday);
        if (rc < 0) {
            taken = -1;
            goto out;
        }
        if (rc == 0)
            break; /* dt <= 0: the reference loop would not advance */
        taken++;
        if (p->steps <= 0 && acc->t <= t_before)
            break;
    }
    acc->V = or_volume_land(nr, nc, h, mask, p->dx);
out:
    free(w.Qx);
    free(w.Qy);
    free(w.Qd1);
    free(w.Qd2);
    free(w.Qop);
    free(w.s);
    return taken;
}
