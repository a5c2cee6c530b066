/*
 * CPU oracle for the FloodCA weighted-cellular-automata (WCA) flood step.
 *
 * TEST INFRASTRUCTURE ONLY. This is a plain-C restatement of the reference
 * algorithm (FloodCA src/kernels/physics.h, src/common/model.c and
 * src/common/rain.c) used to check the CUDA path. Nothing in the product
 * library links, loads or calls it; only tests/, __graft_entry__.smoke() and
 * bench.py's cpu_baseline leg do.
 *
 * Build with -ffp-contract=off so that every float operation rounds once, as
 * in the reference's parity build. Define ORACLE_DOUBLE for the FP64 variant
 * (the reference's FCA_DOUBLE build).
 *
 * Parity pins: tests/test_oracle_golden.py checks this restatement against
 * fixtures produced by the reference itself (compiled from its own sources by
 * oracle/Makefile.ref into oracle/_ref/, see tests/golden/make_golden.py).
 */
#ifndef WCA_ORACLE_H
#define WCA_ORACLE_H

#include <stdint.h>

#ifdef ORACLE_DOUBLE
typedef double oreal;
#else
typedef float oreal;
#endif

enum { OR_LAND = 0, OR_SEA = 1, OR_WALL = 2 };

/* Run parameters. Fields that the reference stores as `real` are rounded to
 * oreal before use so that the float oracle sees the same values as the
 * reference float build (FloodCA src/common/fca_types.h:34-86). */
typedef struct OrParams {
    double dx, g, alpha, tau_h, tau_l, z_sea, dt_max, dt_min, S_bnd;
    int U, K, boundary;               /* boundary: 0 open, 1 closed */
    int edge_n, edge_s, edge_w, edge_e;
    double T_sim, out_every;
    int hyeto;                        /* 0 triangle, 1 uniform */
    double D_h, phi, lambda;
    /* Extensions without a reference counterpart:
     * rain_end > 0 makes the rain source zero for steps starting at
     * t >= rain_end and adds rain_end as a step event; inflow_cell >= 0 adds a
     * triangular point hydrograph (0 at t=0, peak at inflow_t_peak, 0 at
     * inflow_t_end) to that LAND cell after the clamp, before hmax. */
    double rain_end;
    long long inflow_cell;
    double inflow_peak, inflow_t_peak, inflow_t_end;
    int steps;                        /* > 0: fixed step count */
    int n_force_days;                 /* > 0: Rday comes from force_rday[day] */
} OrParams;

typedef struct OrAcc {
    double V, V0, V_rain, V_sea, V_bnd, clamp_err, V_in;
    long long cap_active, cap_total, dt_min_hits;
    double t;
    int step;
    double dt_base;                   /* the oreal value, widened */
    int force_day;
} OrAcc;

/* Reference parity helpers, exported for unit tests. */
double or_hyeto_integral(const OrParams *p, double t, double dt);
double or_next_event_time(const OrParams *p, double t);
double or_inflow_volume(const OrParams *p, double t, double dt);
oreal or_cbrt_sq(oreal hf);
oreal or_face_flux(oreal za, oreal ha, oreal na, uint8_t ma, oreal zb, oreal hb, oreal nb,
                   uint8_t mb, oreal d, oreal w, oreal dt, int K, oreal A, const OrParams *p,
                   int *cap);

/* Initialises acc (V0 from h) exactly like fca_acc_init. */
void or_acc_init(OrAcc *acc, int nr, int nc, const oreal *h, const uint8_t *mask, double dx);

/* Runs at most max_calls steps of the run loop (fca_run semantics, FloodCA
 * src/common/model.c:607-643) and returns the number of steps taken. Rday is
 * read and (with forcing days) overwritten in place. force_rday holds
 * n_force_days raw fields (before lambda) of nr*nc values, or NULL. */
int or_run(int nr, int nc, const oreal *z, oreal *h, const oreal *n, const oreal *C, oreal *Rday,
           const uint8_t *mask, oreal *hmax, oreal *tmax, const OrParams *p, OrAcc *acc,
           int max_calls, const oreal *force_rday);

/* LAND volume sum(h*A) in double (FloodCA src/common/grid.c:125-141). */
double or_volume_land(int nr, int nc, const oreal *h, const uint8_t *mask, double dx);

/* Mass balance error (FloodCA src/common/diag.c:5-14) with the point inflow
 * counted as a source. */
double or_mass_error(const OrAcc *acc);

int or_real_size(void);

#endif
