// Drop-in replacement for FloodCA's CUDA backend entry points
// (src/cuda/cuda_backend.h:14-32), built on the fcab_* sessions.
//
// Compiled twice: without FCA_DOUBLE into libfloodca_b200.so (float `real`)
// and with it into libfloodca_b200_f64.so, matching the caller's build.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <vector>

#include "floodca_b200.h"

namespace {

double now_s()
{
    timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

#ifdef FCA_DOUBLE
constexpr int kPrec = FCAB_PREC_F64;
#else
constexpr int kPrec = FCAB_PREC_F32;
#endif

// Same block check as the reference (src/cuda/kernels.cu:634-638); the block
// shape does not change this implementation's launch, which is strip based.
bool block_ok(const FcaRunCfg *cfg)
{
    if ((cfg->block_x * cfg->block_y) % 32 != 0 || cfg->block_x * cfg->block_y > 1024) {
        fprintf(stderr, "block %dx%d must be a multiple of 32 threads and at most 1024\n",
                cfg->block_x, cfg->block_y);
        return false;
    }
    return true;
}

void to_config(const FcaGrid *g, const FcaRunCfg *cfg, FcabConfig *c)
{
    const FcaPhys &p = cfg->phys;
    fcab_config_defaults(c, g->nrows, g->ncols);
    c->precision = kPrec;
    c->math = FCAB_MATH_EXACT;
    c->K = p.K;
    c->U = p.U;
    c->boundary = p.boundary;
    c->edge_n = g->edge_n;
    c->edge_s = g->edge_s;
    c->edge_w = g->edge_w;
    c->edge_e = g->edge_e;
    c->hyeto = cfg->hyeto;
    c->max_steps = cfg->steps;
    c->dx = (double)p.dx;
    c->g = (double)p.g;
    c->alpha = (double)p.alpha;
    c->tau_h = (double)p.tau_h;
    c->tau_l = (double)p.tau_l;
    c->z_sea = (double)p.z_sea;
    c->dt_max = (double)p.dt_max;
    c->dt_min = (double)p.dt_min;
    c->S_bnd = (double)p.S_bnd;
    c->T_sim = (double)cfg->T_sim;
    c->out_every = (double)cfg->out_every;
    c->D_h = (double)cfg->D_h;
    c->phi = (double)cfg->phi;
}

void report(const char *where)
{
    fprintf(stderr, "floodca_b200: %s: %s\n", where, fcab_last_error());
}

// Reads a float32 raster of n cells into Rday (as `real`) and scales it by
// lambda, like fca_grid_load_rday plus the lambda step of fca_step
// (src/common/grid.c:239-254, src/common/model.c:338-357).
int load_rday(FcaGrid *g, const char *path, real lambda)
{
    const size_t n = (size_t)g->nrows * (size_t)g->ncols;
    FILE *fp = path && path[0] ? fopen(path, "rb") : nullptr;
    if (!fp) {
        fprintf(stderr, "Rday missing: %s\n", path ? path : "(null)");
        return -1;
    }
    std::vector<float> tmp(n);
    const size_t got = fread(tmp.data(), sizeof(float), n, fp);
    fclose(fp);
    if (got != n) {
        fprintf(stderr, "failed to read Rday %s\n", path);
        return -1;
    }
    for (size_t i = 0; i < n; i++) {
        g->Rday[i] = (real)tmp[i];
        if (lambda != (real)1)
            g->Rday[i] *= lambda;
    }
    return 0;
}

// Drives a session to the end of the run, serving pauses: forcing-day
// reloads, progress lines and the ensemble poll hook.
int drive(FcabSim *s, FcaGrid *g, const FcaRunCfg *cfg, FcaAcc *acc, FcaTimers *tm,
          void (*poll)(void *), void *pctx, int poll_every, double t_wall0)
{
    int chunk = 32;
    for (;;) {
        if (fcab_sim_advance(s, chunk) != 0)
            return -2;
        FcabPoll p;
        if (fcab_sim_poll(s, &p) != 0)
            return -2;
        if (p.done)
            return 0;
        if (!p.pause) {
            if (chunk < 256)
                chunk *= 2;
            continue;
        }
        chunk = 32;
        int day = p.force_day;
        if (cfg->n_force_days > 0) {
            int d = p.t < 0.0 ? 0 : (int)(p.t / FCA_DAY_S);
            if (d >= cfg->n_force_days)
                d = cfg->n_force_days - 1;
            if (d != p.force_day) {
                const double ti = now_s();
                if (load_rday(g, cfg->force_files[d], cfg->lambda) != 0) {
                    acc->t = (double)cfg->T_sim;
                    return 1;   // the reference stops the run here
                }
                if (tm)
                    tm->t_io += now_s() - ti;
                const double th = now_s();
                if (fcab_sim_set_rain(s, nullptr, g->Rday) != 0)
                    return -2;
                if (tm)
                    tm->t_h2d += now_s() - th;
                day = d;
            }
        }
        if (poll && poll_every > 0 && p.step > 0 && p.step % poll_every == 0)
            poll(pctx);
        if (!poll && cfg->progress_every > 0 && p.step > 0 && p.step % cfg->progress_every == 0) {
            FcabStats st;
            if (fcab_sim_stats(s, &st) != 0)
                return -2;
            printf("progress step=%d t=%.1f dt_base=%.4g V=%.6e V_rain=%.6e wall=%.1f\n",
                   acc->step + (st.step - acc->step), st.t, st.dt_base, st.V,
                   acc->V_rain + st.V_rain, now_s() - t_wall0);
            fflush(stdout);
        }
        if (fcab_sim_resume(s, day) != 0)
            return -2;
    }
}

// Adds the session's run totals to the reference accumulators.
int collect(FcabSim *s, FcaAcc *acc, int step0)
{
    FcabStats st;
    if (fcab_sim_stats(s, &st) != 0)
        return -2;
    acc->V_rain += st.V_rain;
    acc->clamp_err += st.clamp_err;
    acc->V_sea += st.V_sea;
    acc->V_bnd += st.V_bnd;
    acc->cap_active += (long)st.cap_active;
    acc->cap_total += (long)st.cap_total;
    acc->dt_min_hits += (long)st.dt_min_hits;
    acc->V = st.V;
    acc->t = st.t;
    acc->step = st.step;
    acc->dt_base = (real)st.dt_base;
    (void)step0;
    return 0;
}

}  // namespace

extern "C" void fca_cuda_device_name(char *name, size_t n)
{
    cudaDeviceProp prop;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&prop, dev) != cudaSuccess) {
        snprintf(name, n, "unknown");
        return;
    }
    snprintf(name, n, "%s", prop.name);
}

extern "C" int fca_cuda_select_device(int local_rank)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0)
        return -1;
    const int dev = local_rank % n;
    if (cudaSetDevice(dev) != cudaSuccess)
        return -1;
    return dev;
}

extern "C" int fca_cuda_run(FcaGrid *g, FcaRunCfg *cfg, FcaAcc *acc, FcaTimers *tm)
{
    if (!block_ok(cfg))
        return -1;
    if (!cfg->reduce_impl[0])
        snprintf(cfg->reduce_impl, sizeof(cfg->reduce_impl), "fused");
    FcabConfig c;
    to_config(g, cfg, &c);
    double ti = now_s();
    FcabSim *s = nullptr;
    if (fcab_sim_create(&s, &c, nullptr) != 0) {
        report("create");
        return -2;
    }
    tm->t_init += now_s() - ti;
    ti = now_s();
    if (fcab_sim_upload(s, g->z, g->h, g->n, g->C, g->Rday, g->mask, g->hmax, g->tmax) != 0 ||
        fcab_sim_set_pause_every(s, cfg->progress_every, cfg->n_force_days) != 0 ||
        fcab_sim_reset_time(s, acc->t, acc->step, (double)acc->dt_base, acc->force_day) != 0) {
        report("upload");
        fcab_sim_destroy(s);
        return -2;
    }
    tm->t_h2d = now_s() - ti;
    tm->t_d2h = 0;
    // The step is one fused kernel; the reference's per-phase timers do not apply.
    tm->t_dt = tm->t_flux = tm->t_limiter = tm->t_update = -1;

    const int step0 = acc->step;
    const double t_wall0 = now_s();
    int rc = drive(s, g, cfg, acc, tm, nullptr, nullptr, 0, t_wall0);
    if (rc < 0) {
        report("run");
        fcab_sim_destroy(s);
        return -2;
    }
    FcabPoll p;
    if (fcab_sim_poll(s, &p) != 0) {
        report("run");
        fcab_sim_destroy(s);
        return -2;
    }
    tm->wall_total += now_s() - t_wall0;
    if (collect(s, acc, step0) != 0) {
        report("stats");
        fcab_sim_destroy(s);
        return -2;
    }
    if (rc == 1)
        acc->t = (double)cfg->T_sim;   // a forcing day failed to load: the run ends there
    acc->force_day = p.force_day;
    ti = now_s();
    if (fcab_sim_download(s, g->h, g->hmax, g->tmax) != 0) {
        report("download");
        fcab_sim_destroy(s);
        return -2;
    }
    tm->t_d2h = now_s() - ti;
    fcab_sim_destroy(s);
    // a forcing day failed to load: the state is where the run stopped (as
    // the reference leaves it), but the caller is told
    return rc == 1 ? -3 : 0;
}

// ---------------------------------------------------------------------------
// Ensemble session (src/cuda/kernels.cu:790-1043).

struct FcaCudaEns {
    FcabSim *s;
    int nthr;
    double thr[4];
    size_t N;
    uint16_t *counts;   // device, nthr * N
};

extern "C" FcaCudaEns *fca_cuda_ens_open(const FcaGrid *g, FcaRunCfg *cfg, int nthr,
                                         const double *thr)
{
    if (nthr < 1 || nthr > 4) {
        fprintf(stderr, "fca_cuda_ens_open: %d thresholds, at most %d\n", nthr, 4);
        return nullptr;
    }
    if (!block_ok(cfg))
        return nullptr;
    if (!cfg->reduce_impl[0])
        snprintf(cfg->reduce_impl, sizeof(cfg->reduce_impl), "fused");
    FcaCudaEns *e = (FcaCudaEns *)calloc(1, sizeof(FcaCudaEns));
    if (!e)
        return nullptr;
    e->nthr = nthr;
    for (int j = 0; j < nthr; j++)
        e->thr[j] = thr[j];
    e->N = (size_t)g->nrows * (size_t)g->ncols;
    FcabConfig c;
    to_config(g, cfg, &c);
    if (fcab_sim_create(&e->s, &c, nullptr) != 0 ||
        fcab_sim_upload(e->s, g->z, g->h, g->n, g->C, g->Rday, g->mask, g->hmax, g->tmax) != 0 ||
        cudaMalloc(&e->counts, (size_t)nthr * e->N * sizeof(uint16_t)) != cudaSuccess ||
        cudaMemset(e->counts, 0, (size_t)nthr * e->N * sizeof(uint16_t)) != cudaSuccess) {
        report("ens_open");
        fca_cuda_ens_close(e);
        return nullptr;
    }
    return e;
}

extern "C" int fca_cuda_ens_run(FcaCudaEns *e, FcaGrid *g, const FcaRunCfg *cfg, FcaAcc *acc,
                                FcaTimers *tm, long *flooded, double *max_depth,
                                void (*poll)(void *), void *pctx, int poll_every)
{
    FcabConfig c;
    to_config(g, cfg, &c);
    double ti = now_s();
    if (fcab_sim_set_config(e->s, &c) != 0 || fcab_sim_set_rain(e->s, nullptr, g->Rday) != 0 ||
        fcab_sim_upload_state(e->s, g->h, g->hmax, g->tmax) != 0 ||
        fcab_sim_set_pause_every(e->s, poll ? poll_every : 0, cfg->n_force_days) != 0 ||
        fcab_sim_reset_time(e->s, acc->t, acc->step, (double)acc->dt_base, acc->force_day) != 0) {
        report("ens_run upload");
        return -2;
    }
    tm->t_h2d += now_s() - ti;
    tm->t_dt = tm->t_flux = tm->t_limiter = tm->t_update = -1;
    const int step0 = acc->step;
    const double t_wall0 = now_s();
    const int rc = drive(e->s, g, cfg, acc, tm, poll, pctx, poll_every, t_wall0);
    if (rc < 0) {
        report("ens_run");
        return -2;
    }
    FcabPoll p;
    if (fcab_sim_poll(e->s, &p) != 0)
        return -2;
    tm->wall_total += now_s() - t_wall0;
    if (collect(e->s, acc, step0) != 0)
        return -2;
    if (rc == 1)
        acc->t = (double)cfg->T_sim;
    acc->force_day = p.force_day;
    ti = now_s();
    long long fl[4] = {0, 0, 0, 0};
    if (fcab_sim_count_flooded(e->s, e->nthr, e->thr, e->counts, fl, max_depth) != 0) {
        report("ens_run count");
        return -2;
    }
    tm->t_d2h += now_s() - ti;
    for (int j = 0; j < e->nthr; j++)
        flooded[j] = (long)fl[j];
    return rc == 1 ? -3 : 0;
}

extern "C" int fca_cuda_ens_counts(FcaCudaEns *e, uint16_t *host)
{
    if (cudaMemcpy(host, e->counts, (size_t)e->nthr * e->N * sizeof(uint16_t),
                   cudaMemcpyDeviceToHost) != cudaSuccess)
        return -2;
    return 0;
}

extern "C" void fca_cuda_ens_close(FcaCudaEns *e)
{
    if (!e)
        return;
    if (e->counts)
        cudaFree(e->counts);
    fcab_sim_destroy(e->s);
    free(e);
}
