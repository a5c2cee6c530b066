// Device-resident WCA simulation sessions (the fcab_* C-ABI).
//
// A session owns the padded device layout of one grid (see GridD in
// wca_kernels.cuh), a control block (Ctl) that the kernels advance on their
// own, and CUDA graphs of GRAPH_STEPS step launches that are replayed to
// advance a run. The host only looks at the control block between chunks, to
// end the run or to serve a pause (forcing-day reload, progress line).
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "floodca_b200.h"
#include "wca_dispatch.h"
#include "wca_sim_internal.h"

using namespace fcab;

namespace {

thread_local std::string g_err;

int fail(int code, const char *fmt, ...) __attribute__((format(printf, 2, 3)));
int fail(int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

#define CUDA_TRY(x)                                                                        \
    do {                                                                                   \
        cudaError_t e_ = (x);                                                              \
        if (e_ != cudaSuccess)                                                             \
            return fail(FCAB_ERR_CUDA, "%s:%d %s: %s", __FILE__, __LINE__, #x,             \
                        cudaGetErrorString(e_));                                           \
    } while (0)

constexpr int GRAPH_STEPS = 32;

__global__ void k_fill_interior(void *p, long long pitch, int r_lo, int nr, int nc, double v,
                                int esize)
{
    const long long N = (long long)nr * nc;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N;
         i += (long long)gridDim.x * blockDim.x) {
        const long long a = (r_lo + i / nc + PADR) * pitch + i % nc + PADC;
        if (esize == 8)
            static_cast<double *>(p)[a] = v;
        else
            static_cast<float *>(p)[a] = (float)v;
    }
}

__global__ void k_fill_all(void *p, long long n, double v, int esize)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        if (esize == 8)
            static_cast<double *>(p)[i] = v;
        else
            static_cast<float *>(p)[i] = (float)v;
    }
}

// Writes C*Rday (rounded in the element type, as the reference's
// C[a]*Rday[a]*F multiplies left to right) into the padded field `cr` and
// tracks the minimum and maximum over LAND cells as order-preserving keys,
// so a uniform field can be detected exactly.
template <typename T>
__global__ void k_make_cr(const T *C, const T *R, const uint8_t *m, T *cr, long long pitch,
                          int r_lo, int nr, int nc, unsigned long long *mm, const T *z,
                          const T *h, const T *n)
{
    unsigned long long lo = ~0ull, hi = 0ull, bad = ~0ull;
    const long long N = (long long)nr * nc;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N;
         i += (long long)gridDim.x * blockDim.x) {
        const int r = r_lo + (int)(i / nc), c = (int)(i % nc);
        const long long a = (long long)(r + PADR) * pitch + c + PADC;
        // rain falls on LAND cells only; other cells keep 0 whatever C and
        // Rday hold there
        const T v = m[a] == M_LAND ? C[a] * R[a] : T(0);
        cr[a] = v;
        if (m[a] == M_LAND) {
            unsigned long long key;
            if (sizeof(T) == 4) {
                unsigned b = __float_as_uint((float)v);
                key = (b & 0x80000000u) ? (unsigned long long)(~b) : (unsigned long long)(b | 0x80000000u);
            } else {
                unsigned long long b = (unsigned long long)__double_as_longlong((double)v);
                key = (b >> 63) ? ~b : (b | 0x8000000000000000ull);
            }
            lo = key < lo ? key : lo;
            hi = key > hi ? key : hi;
            // first non-finite input of a LAND cell: 8 * cell + field
            // (0 z, 1 h, 2 n, 3 C, 4 Rday); z, h, n only when given
            int f = -1;
            if (z && !isfinite(z[a]))
                f = 0;
            else if (z && !isfinite(h[a]))
                f = 1;
            else if (z && !isfinite(n[a]))
                f = 2;
            else if (!isfinite(C[a]))
                f = 3;
            else if (!isfinite(R[a]))
                f = 4;
            if (f >= 0 && bad == ~0ull)
                bad = (unsigned long long)i * 8 + f;
        }
    }
    atomicMin(&mm[0], lo);
    atomicMax(&mm[1], hi);
    if (bad != ~0ull)
        atomicMin(&mm[2], bad);
}

size_t esize_of(int prec) { return prec == FCAB_PREC_F64 ? 8 : 4; }

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    });
    return fn;
}

// Row-tile maps of the padded FP32 fields z, n, h0, h1 for the pair sweep's
// TMA row source: 2-D [rows][pitch] floats, boxes of 64 columns x TMA_RB
// rows; rows past the array read as zeros (never used).
bool make_row_maps(FcabSim *s)
{
    auto fn = tensor_map_encoder();
    if (!fn || s->esize != 4)
        return false;
    CUtensorMap maps[4];
    const void *fields[4] = {s->z, s->n, s->h0, s->h1};
    cuuint64_t dims[2] = {(cuuint64_t)s->pitch, (cuuint64_t)s->rows_alloc};
    cuuint64_t strides[1] = {(cuuint64_t)s->pitch * 4};
    cuuint32_t box[2] = {64, (cuuint32_t)TMA_RB};
    cuuint32_t es[2] = {1, 1};
    for (int q = 0; q < 4; q++) {
        if (((uintptr_t)fields[q] & 15) ||
            fn(&maps[q], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, (void *)fields[q], dims, strides, box,
               es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
               CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) !=
                CUDA_SUCCESS)
            return false;
    }
    if (fcab::cached_malloc(&s->tmaps, sizeof(maps)) != cudaSuccess)
        return false;
    return cudaMemcpyAsync(s->tmaps, maps, sizeof(maps), cudaMemcpyHostToDevice, s->stream) ==
           cudaSuccess;
}

// Row source of the FP32 pair sweep: FCAB_ROW_SOURCE=tma streams rows by
// TMA into shared memory, anything else (the default) by plain loads.
bool want_tma_rows()
{
    const char *e = getenv("FCAB_ROW_SOURCE");
    return e && strcmp(e, "tma") == 0;
}

}  // namespace

namespace fcab {

void set_error(const char *msg) { g_err = msg; }

}  // namespace fcab

extern "C" const char *fcab_last_error(void) { return g_err.c_str(); }

extern "C" const char *fcab_version(void) { return "floodca_b200 0.1 sm_100a"; }

extern "C" void fcab_config_defaults(FcabConfig *c, int nrows, int ncols)
{
    memset(c, 0, sizeof(*c));
    c->nrows = nrows;
    c->ncols = ncols;
    c->precision = FCAB_PREC_F32;
    c->math = FCAB_MATH_EXACT;
    c->K = 4;
    c->U = 1;
    c->boundary = FCA_BND_OPEN;
    c->edge_n = c->edge_s = c->edge_w = c->edge_e = 1;
    c->hyeto = FCA_HYETO_TRIANGLE;
    c->max_steps = 0;
    c->dx = 30.0;
    c->g = 9.81;
    c->alpha = 0.5;
    c->tau_h = 1e-3;
    c->tau_l = 1e-5;
    c->z_sea = 0.0;
    c->dt_max = 60.0;
    c->dt_min = 0.01;
    c->S_bnd = 0.001;
    c->T_sim = 86400.0;
    c->out_every = 0.0;
    c->D_h = 24.0;
    c->phi = 0.5;
    c->rain_end = 0.0;
    c->inflow_cell = -1;
    c->cols_per_lane = 0;
    c->seg_rows = 0;
}

// ---------------------------------------------------------------------------

static double as_real(double v, int prec) { return prec == FCAB_PREC_F64 ? v : (double)(float)v; }

// hn, hs: halo rows above and below a slab's own rows; the inflow cell then
// indexes the uploaded (hn + nrows + hs) x ncols array.
template <typename T>
static void fill_runk(RunK<T> &rk, const FcabConfig &c, int hn = 0, int hs = 0)
{
    memset(&rk, 0, sizeof(rk));
    StepK<T> &k = rk.k;
    k.dx = (T)c.dx;
    k.A = k.dx * k.dx;
    k.g = (T)c.g;
    k.tau_h = (T)c.tau_h;
    k.tau_l = (T)c.tau_l;
    k.z_sea = (T)c.z_sea;
    k.S_bnd = (T)c.S_bnd;
    // physics.h:37-48: ((real)sqrt(2.0) - 1) * dx and (real)sqrt(2.0) * dx
    const T sq2 = (T)std::sqrt(2.0);
    k.w = c.K == 8 ? (sq2 - T(1)) * k.dx : k.dx;
    k.d_diag = sq2 * k.dx;
    k.rdx = T(1) / k.dx;
    k.rdd = T(1) / k.d_diag;
    k.alpha_dx = (T)c.alpha * k.dx;
    k.inv_A = T(1) / k.A;
    rk.dt_max = (T)c.dt_max;
    rk.dt_min = (T)c.dt_min;
    rk.K = c.K;
    rk.U = c.U > 0 ? c.U : 1;
    rk.open = c.boundary == FCA_BND_OPEN;
    rk.edge_n = c.edge_n;
    rk.edge_s = c.edge_s;
    rk.edge_w = c.edge_w;
    rk.edge_e = c.edge_e;
    rk.inflow_r = rk.inflow_c = -1;
    if (c.inflow_cell >= 0 && c.inflow_cell < (long long)(c.nrows + hn + hs) * c.ncols) {
        rk.inflow_r = (int)(c.inflow_cell / c.ncols) - hn;
        rk.inflow_c = (int)(c.inflow_cell % c.ncols);
    }
}

int fcab::pick_cpl(const FcabConfig &c)
{
    if (c.cols_per_lane == 1 || c.cols_per_lane == 2 || c.cols_per_lane == 4)
        return c.cols_per_lane;
    // 1-column lanes for grids too small to fill the GPU with 2-column
    // strips (measured on a B200: CPL 1 is faster up to 1024^2, CPL 2 from
    // 2048^2 on, where its smaller halo share wins)
    const long long strips2 = (c.ncols + 55) / 56;
    if (c.ncols <= 64 || strips2 * c.nrows < 40960)
        return 1;
    return 2;
}

long long fcab::step_warps(const FcabConfig &c, int cpl, int nsm, int per_sm, int wpb)
{
    const int ow = 32 * cpl - 2 * (cpl == 1 ? 3 : 4);
    const long long strips = (c.ncols + ow - 1) / ow;
    const long long total = strips * c.nrows;
    const long long max_warps = (long long)nsm * (per_sm > 0 ? per_sm : 1) * wpb;
    // rows per warp: enough warps to fill the resident slots, but at least 4
    // rows per warp (each warp's segment costs 6 extra pipeline rows)
    long long seg = c.seg_rows > 0 ? c.seg_rows : total / max_warps;
    if (seg < 4)
        seg = 4;
    const long long want = (total + seg - 1) / seg;
    const long long warps = want < max_warps ? want : max_warps;
    return warps < 1 ? 1 : warps;
}

// Rejects configurations the step cannot run: unknown enumerations, a dt
// reuse count below 1, non-positive or non-finite cell size, gravity,
// Courant factor or dt bounds (a zero dt never advances the clock), negative
// thresholds, non-finite times and unsupported launch overrides. Makes no
// CUDA call.
static int validate_config(const FcabConfig *c)
{
    auto pos = [](double v) { return std::isfinite(v) && v > 0.0; };
    auto nonneg = [](double v) { return std::isfinite(v) && v >= 0.0; };
    if (c->nrows < 1 || c->ncols < 1)
        return fail(FCAB_ERR_ARG, "grid %dx%d is empty", c->nrows, c->ncols);
    if ((long long)c->nrows * c->ncols > (1ll << 40))
        return fail(FCAB_ERR_ARG, "grid too large");
    if (c->K != 4 && c->K != 8)
        return fail(FCAB_ERR_ARG, "K=%d: only 4 or 8 neighbours", c->K);
    if (c->precision < FCAB_PREC_F32 || c->precision > FCAB_PREC_F64)
        return fail(FCAB_ERR_ARG, "unknown precision %d", c->precision);
    if (c->math != FCAB_MATH_EXACT && c->math != FCAB_MATH_FAST)
        return fail(FCAB_ERR_ARG, "unknown math mode %d", c->math);
    if (c->U < 1)
        return fail(FCAB_ERR_ARG, "U=%d: the dt reuse count is at least 1", c->U);
    if (c->boundary != FCA_BND_OPEN && c->boundary != FCA_BND_CLOSED)
        return fail(FCAB_ERR_ARG, "unknown boundary %d", c->boundary);
    if (c->hyeto != FCA_HYETO_TRIANGLE && c->hyeto != FCA_HYETO_UNIFORM)
        return fail(FCAB_ERR_ARG, "unknown hyetograph %d", c->hyeto);
    if (!pos(c->dx) || !pos(c->g) || !pos(c->alpha))
        return fail(FCAB_ERR_ARG, "dx, g and alpha must be finite and positive");
    if (!pos(c->dt_max) || !pos(c->dt_min))
        return fail(FCAB_ERR_ARG, "dt_max and dt_min must be finite and positive");
    if (!nonneg(c->tau_h) || !nonneg(c->tau_l))
        return fail(FCAB_ERR_ARG, "tau_h and tau_l must be finite and not negative");
    if (!std::isfinite(c->z_sea) || !std::isfinite(c->S_bnd) || !std::isfinite(c->T_sim) ||
        !std::isfinite(c->out_every) || !std::isfinite(c->D_h) || !std::isfinite(c->phi) ||
        !std::isfinite(c->rain_end))
        return fail(FCAB_ERR_ARG, "z_sea, S_bnd, T_sim, out_every, D_h, phi and rain_end must be finite");
    if (c->max_steps < 0)
        return fail(FCAB_ERR_ARG, "max_steps=%d is negative", c->max_steps);
    if (c->cols_per_lane != 0 && c->cols_per_lane != 1 && c->cols_per_lane != 2 &&
        c->cols_per_lane != 4)
        return fail(FCAB_ERR_ARG, "cols_per_lane=%d: 0, 1, 2 or 4", c->cols_per_lane);
    if (c->seg_rows < 0)
        return fail(FCAB_ERR_ARG, "seg_rows=%d is negative", c->seg_rows);
    if (c->inflow_cell >= 0 && (!std::isfinite(c->inflow_peak) || !std::isfinite(c->inflow_t_peak) ||
                                !std::isfinite(c->inflow_t_end)))
        return fail(FCAB_ERR_ARG, "inflow hydrograph values must be finite");
    return FCAB_OK;
}

extern "C" int fcab_sim_create(FcabSim **out, const FcabConfig *cfg, void *stream)
{
    *out = nullptr;
    if (int rc = validate_config(cfg))
        return rc;

    FcabSim *s = new FcabSim();
    s->cfg = *cfg;
    s->cpl = pick_cpl(*cfg);
    s->esize = esize_of(cfg->precision);
    cudaError_t e = cudaGetDevice(&s->dev);
    if (e != cudaSuccess) {
        delete s;
        return fail(FCAB_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
    }
    if (stream) {
        s->stream = (cudaStream_t)stream;
        s->own_stream = false;
    } else {
        e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            delete s;
            return fail(FCAB_ERR_CUDA, "cudaStreamCreate: %s", cudaGetErrorString(e));
        }
        s->own_stream = true;
    }
    // Padded layout: PADR rows above and below, PADC columns left, and at
    // least one strip width of slack right; pitch rounded to 32 elements.
    s->pitch = ((long long)PADC + cfg->ncols + 128 + 31) / 32 * 32;
    s->rows_alloc = cfg->nrows + 2 * PADR;
    s->nelem = (size_t)s->pitch * (size_t)s->rows_alloc;

    const size_t fb = s->nelem * s->esize;
    void **fields[] = {&s->z, &s->n, &s->h0, &s->h1, &s->hmax, &s->tmax};
    for (void **f : fields) {
        e = fcab::cached_malloc(f, fb);
        if (e != cudaSuccess) {
            fcab_sim_destroy(s);
            return fail(FCAB_ERR_CUDA, "cudaMalloc(%zu): %s", fb, cudaGetErrorString(e));
        }
    }
    if ((e = fcab::cached_malloc((void **)&s->m, s->nelem)) != cudaSuccess ||
        (e = fcab::cached_malloc((void **)&s->ctl, sizeof(Ctl))) != cudaSuccess ||
        (e = fcab::cached_malloc(&s->scratch, 64)) != cudaSuccess ||
        (e = fcab::cached_malloc_host(&s->ctl_host, sizeof(Ctl))) != cudaSuccess) {
        fcab_sim_destroy(s);
        return fail(FCAB_ERR_CUDA, "allocation: %s", cudaGetErrorString(e));
    }
    if (cfg->precision != FCAB_PREC_F64 && want_tma_rows())
        s->use_tma = make_row_maps(s);
    if (cfg->precision == FCAB_PREC_F64)
        fill_runk<double>(s->rkd, *cfg);
    else
        fill_runk<float>(s->rkf, *cfg);
    const int p = cfg->precision;
    TimeCfg &tc = s->tc;
    memset(&tc, 0, sizeof(tc));
    tc.T_sim = as_real(cfg->T_sim, p);
    tc.out_every = as_real(cfg->out_every, p);
    tc.D_h = as_real(cfg->D_h, p);
    tc.phi = as_real(cfg->phi, p);
    tc.rain_end = cfg->rain_end;
    tc.inflow_peak = cfg->inflow_peak;
    tc.inflow_t_peak = cfg->inflow_t_peak;
    tc.inflow_t_end = cfg->inflow_t_end;
    tc.hyeto = cfg->hyeto;
    tc.max_steps = cfg->max_steps;
    tc.U = cfg->U > 0 ? cfg->U : 1;
    tc.time_f32 = p == FCAB_PREC_F32_ALL;
    tc.prec_f64 = p == FCAB_PREC_F64;
    tc.vseed_on = 1;        // seeded dt pruning; a missed seed is settled by the full
    tc.tail_vpass = 1;      // velocity pass, which the step kernel launches itself
    *out = s;
    return 0;
}

extern "C" void fcab_sim_destroy(FcabSim *s)
{
    if (!s)
        return;
    if (s->graph)
        cudaGraphExecDestroy(s->graph);
    if (s->stream)
        cudaStreamSynchronize(s->stream);
    void *ptrs[] = {s->z, s->n, s->cr, s->h0, s->h1, s->hmax, s->tmax, s->m, s->ctl,
                    s->scratch, s->tmpC, s->tmpR, s->tmaps};
    for (void *q : ptrs)
        if (q)
            fcab::cached_free(q);
    if (s->ctl_host)
        fcab::cached_free(s->ctl_host);
    if (s->own_stream && s->stream)
        cudaStreamDestroy(s->stream);
    delete s;
}

// Copies a row-major nrows x ncols array (host or device) into the interior of
// a padded field; a slab's arrays carry its halo rows too.
static cudaError_t put_field(FcabSim *s, void *dst, const void *src, size_t esz,
                             cudaMemcpyKind kind)
{
    char *d = (char *)dst + ((size_t)(PADR - s->hn) * s->pitch + PADC) * esz;
    const size_t rows = (size_t)(s->cfg.nrows + s->hn + s->hs);
    if (kind == cudaMemcpyHostToDevice)
        return fcab::h2d_rows(d, (size_t)s->pitch * esz, src, (size_t)s->cfg.ncols * esz, rows,
                              s->stream);
    return cudaMemcpy2DAsync(d, (size_t)s->pitch * esz, src, (size_t)s->cfg.ncols * esz,
                             (size_t)s->cfg.ncols * esz, rows, kind, s->stream);
}

static cudaError_t get_field(FcabSim *s, void *dst, const void *src, size_t esz)
{
    const char *sp = (const char *)src + ((size_t)PADR * s->pitch + PADC) * esz;
    return fcab::d2h_rows(dst, sp, (size_t)s->pitch * esz, (size_t)s->cfg.ncols * esz,
                          (size_t)s->cfg.nrows, s->stream);
}

static int fill_interior(FcabSim *s, void *dst, double v)
{
    // Padding stays zero; the nrows x ncols interior gets v.
    CUDA_TRY(cudaMemsetAsync(dst, 0, s->nelem * s->esize, s->stream));
    k_fill_interior<<<1024, 256, 0, s->stream>>>(dst, s->pitch, -s->hn,
                                                 s->cfg.nrows + s->hn + s->hs, s->cfg.ncols, v,
                                                 (int)s->esize);
    CUDA_TRY(cudaGetLastError());
    return 0;
}

// Rebuilds cr = C*Rday from the staging copies tmpC/tmpR (padded layout)
// and decides whether the field is uniform over LAND cells. Fails with
// FCAB_ERR_ARG when a LAND cell's C or Rday (and, with check_state, its z,
// h or n) is not finite.
static int rebuild_rain(FcabSim *s, bool check_state)
{
    unsigned long long init[3] = {~0ull, 0ull, ~0ull};
    CUDA_TRY(cudaMemcpyAsync(s->scratch, init, sizeof(init), cudaMemcpyHostToDevice, s->stream));
    if (!s->cr)
        CUDA_TRY(fcab::cached_malloc(&s->cr, s->nelem * s->esize));
    CUDA_TRY(cudaMemsetAsync(s->cr, 0, s->nelem * s->esize, s->stream));
    const int nb = 1024;
    if (s->esize == 8)
        k_make_cr<double><<<nb, 256, 0, s->stream>>>(
            (const double *)s->tmpC, (const double *)s->tmpR, s->m, (double *)s->cr, s->pitch,
            -s->hn, s->cfg.nrows + s->hn + s->hs, s->cfg.ncols, (unsigned long long *)s->scratch,
            check_state ? (const double *)s->z : nullptr, (const double *)s->h0,
            (const double *)s->n);
    else
        k_make_cr<float><<<nb, 256, 0, s->stream>>>(
            (const float *)s->tmpC, (const float *)s->tmpR, s->m, (float *)s->cr, s->pitch,
            -s->hn, s->cfg.nrows + s->hn + s->hs, s->cfg.ncols, (unsigned long long *)s->scratch,
            check_state ? (const float *)s->z : nullptr, (const float *)s->h0,
            (const float *)s->n);
    CUDA_TRY(cudaGetLastError());
    unsigned long long mm[3];
    CUDA_TRY(cudaMemcpyAsync(mm, s->scratch, sizeof(mm), cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    if (mm[2] != ~0ull) {
        static const char *names[5] = {"z", "h", "n", "C", "Rday"};
        const long long cell = (long long)(mm[2] >> 3);
        return fail(FCAB_ERR_ARG, "%s is not finite at LAND cell (row %lld, col %lld)",
                    names[mm[2] & 7], cell / s->cfg.ncols - s->hn, cell % s->cfg.ncols);
    }
    double uni = 0.0;
    bool uniform = true;
    if (mm[0] != ~0ull) {
        uniform = mm[0] == mm[1];
        unsigned long long key = mm[0];
        if (s->esize == 8) {
            unsigned long long b = (key >> 63) ? (key & 0x7fffffffffffffffull) : ~key;
            double d;
            memcpy(&d, &b, 8);
            uni = d;
        } else {
            unsigned kb = (unsigned)key;
            unsigned b = (kb & 0x80000000u) ? (kb & 0x7fffffffu) : ~kb;
            float f;
            memcpy(&f, &b, 4);
            uni = f;
        }
    }
    s->rain_field = !uniform;
    if (s->esize == 8)
        s->rkd.cr_uniform = uni;
    else
        s->rkf.cr_uniform = (float)uni;
    s->variant_dirty = true;
    return 0;
}

static int upload_common(FcabSim *s, const void *z, const void *h, const void *n, const void *C,
                         const void *Rday, const uint8_t *mask, const void *hmax,
                         const void *tmax, cudaMemcpyKind kind)
{
    const FcabConfig &c = s->cfg;
    const size_t es = s->esize;
    if (!z || !h || !mask)
        return fail(FCAB_ERR_ARG, "z, h and mask are required");
    CUDA_TRY(cudaMemsetAsync(s->z, 0, s->nelem * es, s->stream));
    CUDA_TRY(cudaMemsetAsync(s->h0, 0, s->nelem * es, s->stream));
    CUDA_TRY(cudaMemsetAsync(s->h1, 0, s->nelem * es, s->stream));
    CUDA_TRY(cudaMemsetAsync(s->hmax, 0, s->nelem * es, s->stream));
    CUDA_TRY(cudaMemsetAsync(s->tmax, 0, s->nelem * es, s->stream));
    CUDA_TRY(cudaMemsetAsync(s->m, M_WALL, s->nelem, s->stream));
    CUDA_TRY(put_field(s, s->z, z, es, kind));
    CUDA_TRY(put_field(s, s->h0, h, es, kind));
    CUDA_TRY(put_field(s, s->m, mask, 1, kind));
    if (n) {
        CUDA_TRY(cudaMemsetAsync(s->n, 0, s->nelem * es, s->stream));
        CUDA_TRY(put_field(s, s->n, n, es, kind));
    } else {
        int rc = fill_interior(s, s->n, as_real(0.03, c.precision));
        if (rc)
            return rc;
    }
    CUDA_TRY(put_field(s, s->hmax, hmax ? hmax : h, es, kind));
    if (tmax)
        CUDA_TRY(put_field(s, s->tmax, tmax, es, kind));
    // staging copies of C and Rday for the rain field
    if (!s->tmpC)
        CUDA_TRY(fcab::cached_malloc(&s->tmpC, s->nelem * es));
    if (!s->tmpR)
        CUDA_TRY(fcab::cached_malloc(&s->tmpR, s->nelem * es));
    CUDA_TRY(cudaMemsetAsync(s->tmpC, 0, s->nelem * es, s->stream));
    CUDA_TRY(cudaMemsetAsync(s->tmpR, 0, s->nelem * es, s->stream));
    if (C)
        CUDA_TRY(put_field(s, s->tmpC, C, es, kind));
    if (Rday)
        CUDA_TRY(put_field(s, s->tmpR, Rday, es, kind));
    int rc = rebuild_rain(s, true);
    if (rc)
        return rc;
    // has SEA / inflow cell LAND
    std::vector<uint8_t> probe;
    const long long N = (long long)c.nrows * c.ncols;
    const long long Nup = (long long)(c.nrows + s->hn + s->hs) * c.ncols;   // with halo rows
    const uint8_t *mup = mask;
    if (kind != cudaMemcpyHostToDevice) {
        probe.resize((size_t)Nup);
        CUDA_TRY(cudaMemcpy(probe.data(), mask, (size_t)Nup, cudaMemcpyDeviceToHost));
        mup = probe.data();
    }
    const uint8_t *mh = mup + (long long)s->hn * c.ncols;              // own rows
    const int has_sea = memchr(mup, M_SEA, (size_t)Nup) != nullptr;
    // LAND cells per row; open faces only on the open edges' rows/columns
    s->land_cells = 0;
    s->open_faces = 0;
    const bool open = c.boundary == FCA_BND_OPEN;
    for (long long r = 0; r < c.nrows; r++) {
        const uint8_t *row = mh + r * c.ncols;
        long long cnt = 0;
        for (long long k = 0; k < c.ncols; k++)
            cnt += row[k] == M_LAND;
        s->land_cells += cnt;
        if (open) {
            s->open_faces += (r == 0 && c.edge_n ? cnt : 0) + (r == c.nrows - 1 && c.edge_s ? cnt : 0);
            s->open_faces += (c.edge_w && row[0] == M_LAND) + (c.edge_e && row[c.ncols - 1] == M_LAND);
        }
    }
    // all-LAND grids use the mask-free kernel: padding elevation PAD_Z makes
    // every face to the padding carry zero discharge (needs tau_h > 0)
    long long land_up = s->land_cells;       // with a slab's halo rows
    for (long long k = 0; k < (long long)s->hn * c.ncols; k++)
        land_up += mup[k] == M_LAND;
    for (long long k = N + (long long)s->hn * c.ncols; k < Nup; k++)
        land_up += mup[k] == M_LAND;
    const bool all_land = c.tau_h > 0.0 && s->land_cells == N && land_up == Nup;
    s->landonly = all_land;
    if (all_land) {
        k_fill_all<<<1024, 256, 0, s->stream>>>(s->z, (long long)s->nelem, PAD_Z, (int)es);
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(put_field(s, s->z, z, es, kind));
    }
    int inflow_ok = 0;
    if (c.inflow_cell >= 0 && c.inflow_cell < Nup)
        inflow_ok = mup[c.inflow_cell] == M_LAND;
    const long long nr = c.nrows, nc = c.ncols;
    // a slab also owns the faces between its last row and the south halo
    const long long ny = nr - 1 + (s->hs > 0 ? 1 : 0);
    s->faces_per_step = nr * (nc - 1) + ny * nc + (c.K == 8 ? 2 * ny * (nc - 1) : 0) +
                        s->open_faces;
    if (s->esize == 8) {
        s->rkd.has_sea = has_sea;
    } else {
        s->rkf.has_sea = has_sea;
    }
    s->tc.inflow_ok = inflow_ok;
    s->uploaded = true;
    s->h_cur_host = 0;
    return fcab_sim_reset_time(s, 0.0, 0, 0.0, -1);
}

extern "C" int fcab_sim_upload(FcabSim *s, const void *z, const void *h, const void *n,
                               const void *C, const void *Rday, const uint8_t *mask,
                               const void *hmax, const void *tmax)
{
    return upload_common(s, z, h, n, C, Rday, mask, hmax, tmax, cudaMemcpyHostToDevice);
}

extern "C" int fcab_sim_upload_device(FcabSim *s, const void *z, const void *h, const void *n,
                                      const void *C, const void *Rday, const uint8_t *mask,
                                      const void *hmax, const void *tmax)
{
    return upload_common(s, z, h, n, C, Rday, mask, hmax, tmax, cudaMemcpyDeviceToDevice);
}

extern "C" int fcab_sim_set_rain(FcabSim *s, const void *C, const void *Rday)
{
    if (!s->uploaded)
        return fail(FCAB_ERR_STATE, "set_rain before upload");
    if (C)
        CUDA_TRY(put_field(s, s->tmpC, C, s->esize, cudaMemcpyHostToDevice));
    if (Rday)
        CUDA_TRY(put_field(s, s->tmpR, Rday, s->esize, cudaMemcpyHostToDevice));
    return rebuild_rain(s, false);
}

static int resolve_variant(FcabSim *s)
{
    if (!s->variant_dirty && s->have_variant)
        return 0;
    VariantKey key;
    key.prec = s->cfg.precision;
    key.K = s->cfg.K;
    key.cpl = s->cpl;
    key.math = s->cfg.precision == FCAB_PREC_F32 ? s->cfg.math : FCAB_MATH_EXACT;
    key.rainf = s->rain_field ? 1 : 0;
    key.landonly = s->landonly ? 1 : 0;
    // the pair and four-column sweeps (FP32, all-LAND, two or four columns
    // per lane) address the fields with 32-bit element offsets: larger grids
    // take one column per lane
    if (s->esize == 4 && key.landonly && (key.cpl == 2 || key.cpl == 4) &&
        (long long)(s->cfg.nrows + s->hn + s->hs + 2 * PADR) * s->pitch >= (1ll << 31))
        key.cpl = s->cpl = 1;
    bool ok = key.prec == FCAB_PREC_F32 ? lookup_f32(key, &s->L)
              : key.prec == FCAB_PREC_F32_ALL ? lookup_f32all(key, &s->L)
                                               : lookup_f64(key, &s->L);
    if (!ok)
        return fail(FCAB_ERR_ARG, "no compiled variant prec=%d K=%d cpl=%d math=%d", key.prec,
                    key.K, key.cpl, key.math);
    // Grid: resident CTAs, or fewer so every warp streams >= seg_rows rows.
    int nsm = 0, per_sm = 0;
    CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, s->dev));
    const int smem = s->use_tma ? s->L.tma_smem : 0;
    if (smem > 0)
        CUDA_TRY(cudaFuncSetAttribute(s->L.step_fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      smem));
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, s->L.step_fn, s->L.threads,
                                                           smem));
    if (per_sm < 1)
        per_sm = 1;
    const int wpb = s->L.threads / 32;     // warps per CTA
    s->grid = (int)((step_warps(s->cfg, s->cpl, nsm, per_sm, wpb) + wpb - 1) / wpb);
    s->warps_total = s->grid * wpb;
    s->occupancy = per_sm;
    if (s->graph) {
        cudaGraphExecDestroy(s->graph);
        s->graph = nullptr;
    }
    s->have_variant = true;
    s->variant_dirty = false;
    return 0;
}

template <typename T>
static void grid_view(FcabSim *s, GridD<T> &g)
{
    g.z = (const T *)s->z;
    g.n = (const T *)s->n;
    g.cr = s->rain_field ? (const T *)s->cr : nullptr;
    g.m = s->m;
    g.h0 = (T *)s->h0;
    g.h1 = (T *)s->h1;
    g.hmax = (T *)s->hmax;
    g.tmax = (T *)s->tmax;
    g.pitch = s->pitch;
    g.nr = s->cfg.nrows;
    g.nc = s->cfg.ncols;
    g.r_lo = -s->hn;
    g.r_hi = s->cfg.nrows + s->hs;
    g.tmap = s->use_tma && s->L.tma_smem > 0 ? static_cast<const CUtensorMap *>(s->tmaps)
                                             : nullptr;
}

static int step_smem(const FcabSim *s) { return s->use_tma ? s->L.tma_smem : 0; }

// Host launches per step: the step; with seeded dt pruning and no tail
// launch, also the guarded full velocity pass (it returns at once unless the
// step deferred its dt). A tail-launched pass runs only when the seed missed
// (FcabStats.dt_full_passes counts those).
static int launches_per_step(const FcabSim *s)
{
    return s->tc.vseed_on && !s->tc.tail_vpass ? 2 : 1;
}

static cudaError_t launch_one(FcabSim *s)
{
    const int full_grid = 2 * 148 * 4;
    cudaError_t e;
    if (s->esize == 8) {
        GridD<double> g;
        grid_view(s, g);
        e = s->L.step(&g, &s->rkd, s->tc, s->ctl, s->warps_total, s->grid, s->stream,
                      step_smem(s));
        if (e == cudaSuccess && s->tc.vseed_on && !s->tc.tail_vpass)
            e = s->L.init(&g, &s->rkd, s->tc, s->ctl, full_grid, s->stream, 1);
        return e;
    }
    GridD<float> g;
    grid_view(s, g);
    e = s->L.step(&g, &s->rkf, s->tc, s->ctl, s->warps_total, s->grid, s->stream,
                  step_smem(s));
    if (e == cudaSuccess && s->tc.vseed_on && !s->tc.tail_vpass)
        e = s->L.init(&g, &s->rkf, s->tc, s->ctl, full_grid, s->stream, 1);
    return e;
}

extern "C" int fcab_sim_reset_time(FcabSim *s, double t, int step, double dt_base, int force_day)
{
    if (!s->uploaded)
        return fail(FCAB_ERR_STATE, "reset_time before upload");
    int rc = resolve_variant(s);
    if (rc)
        return rc;
    Ctl c;
    memset(&c, 0, sizeof(c));
    c.t = t;
    c.step = step;
    c.dt_base = dt_base;
    c.force_day = force_day;
    c.h_cur = s->h_cur_host;
    s->step0 = step;
    CUDA_TRY(cudaMemcpyAsync(s->ctl, &c, sizeof(Ctl), cudaMemcpyHostToDevice, s->stream));
    // V0 = LAND volume of the current depth
    double *vol = (double *)s->scratch;
    CUDA_TRY(cudaMemsetAsync(vol, 0, sizeof(double), s->stream));
    if (s->esize == 8) {
        GridD<double> g;
        grid_view(s, g);
        k_volume<double><<<512, 256, 0, s->stream>>>(g, s->ctl, s->rkd.k.A, vol);
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(s->L.init(&g, &s->rkd, s->tc, s->ctl, 2 * 148 * 4, s->stream, 0));
    } else {
        GridD<float> g;
        grid_view(s, g);
        k_volume<float><<<512, 256, 0, s->stream>>>(g, s->ctl, s->rkf.k.A, vol);
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(s->L.init(&g, &s->rkf, s->tc, s->ctl, 2 * 148 * 4, s->stream, 0));
    }
    s->launches += 2;
    CUDA_TRY(cudaMemcpyAsync(&s->V0, vol, sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    s->inited = true;
    return 0;
}

static int ensure_graph(FcabSim *s)
{
    if (s->graph)
        return 0;
    cudaGraph_t g;
    CUDA_TRY(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t le = cudaSuccess;
    for (int i = 0; i < GRAPH_STEPS && le == cudaSuccess; i++)
        le = launch_one(s);
    cudaError_t ee = cudaStreamEndCapture(s->stream, &g);
    if (le != cudaSuccess || ee != cudaSuccess)
        return fail(FCAB_ERR_CUDA, "graph capture: %s / %s", cudaGetErrorString(le),
                    cudaGetErrorString(ee));
    cudaError_t ie = cudaGraphInstantiate(&s->graph, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess)
        return fail(FCAB_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(ie));
    return 0;
}

extern "C" int fcab_sim_advance(FcabSim *s, int nsteps)
{
    if (!s->inited)
        return fail(FCAB_ERR_STATE, "advance before upload");
    if (s->slab)
        return fail(FCAB_ERR_STATE, "a slab steps through fcab_sim_slab_step");
    int rc = resolve_variant(s);
    if (rc)
        return rc;
    if (nsteps >= GRAPH_STEPS) {
        rc = ensure_graph(s);
        if (rc)
            return rc;
    }
    while (nsteps >= GRAPH_STEPS) {
        CUDA_TRY(cudaGraphLaunch(s->graph, s->stream));
        s->launches += GRAPH_STEPS * launches_per_step(s);
        nsteps -= GRAPH_STEPS;
    }
    for (; nsteps > 0; nsteps--) {
        CUDA_TRY(launch_one(s));
        s->launches += launches_per_step(s);
    }
    return 0;
}

// Runs the guarded full velocity pass from the host (it does nothing unless
// a step left its dt deferred).
static int settle_deferred_dt(FcabSim *s)
{
    const int full_grid = 2 * 148 * 4;
    cudaError_t e;
    if (s->esize == 8) {
        GridD<double> g;
        grid_view(s, g);
        e = s->L.init(&g, &s->rkd, s->tc, s->ctl, full_grid, s->stream, 1);
    } else {
        GridD<float> g;
        grid_view(s, g);
        e = s->L.init(&g, &s->rkf, s->tc, s->ctl, full_grid, s->stream, 1);
    }
    CUDA_TRY(e);
    s->launches += 1;
    return 0;
}

extern "C" int fcab_sim_poll(FcabSim *s, FcabPoll *p)
{
    CUDA_TRY(cudaMemcpyAsync(s->ctl_host, s->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    if (((const Ctl *)s->ctl_host)->need_v && !s->slab) {
        // a deferred dt the step's tail launch did not settle (its launch
        // failed): settle it here so the run goes on
        int rc = settle_deferred_dt(s);
        if (rc)
            return rc;
        CUDA_TRY(cudaMemcpyAsync(s->ctl_host, s->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost,
                                 s->stream));
        CUDA_TRY(cudaStreamSynchronize(s->stream));
    }
    const Ctl *c = (const Ctl *)s->ctl_host;
    p->t = c->t;
    p->dt_base = c->dt_base;
    p->step = c->step;
    p->done = c->done;
    p->pause = c->pause;
    p->force_day = c->force_day;
    s->h_cur_host = c->h_cur;
    return 0;
}

extern "C" int fcab_sim_resume(FcabSim *s, int force_day)
{
    // Clears a pause: records the loaded forcing day and re-arms the step.
    Ctl *c = (Ctl *)s->ctl_host;
    CUDA_TRY(cudaMemcpyAsync(s->ctl_host, s->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    c->force_day = force_day;
    c->pause = 0;
    c->active = c->done ? 0 : 1;
    CUDA_TRY(cudaMemcpyAsync(s->ctl, s->ctl_host, sizeof(Ctl), cudaMemcpyHostToDevice, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    return 0;
}

extern "C" int fcab_sim_run(FcabSim *s)
{
    FcabPoll p;
    int chunk = GRAPH_STEPS;
    for (;;) {
        int rc = fcab_sim_advance(s, chunk);
        if (rc)
            return rc;
        rc = fcab_sim_poll(s, &p);
        if (rc)
            return rc;
        if (p.done)
            return 0;
        if (p.pause)
            return fail(FCAB_ERR_STATE, "run paused (forcing or progress); use the drop-in loop");
        if (chunk < 8 * GRAPH_STEPS)
            chunk *= 2;
    }
}

extern "C" int fcab_sim_stats(FcabSim *s, FcabStats *st)
{
    CUDA_TRY(cudaMemcpyAsync(s->ctl_host, s->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s->stream));
    double *vol = (double *)s->scratch;
    CUDA_TRY(cudaMemsetAsync(vol, 0, sizeof(double), s->stream));
    if (s->esize == 8) {
        GridD<double> g;
        grid_view(s, g);
        k_volume<double><<<512, 256, 0, s->stream>>>(g, s->ctl, s->rkd.k.A, vol);
    } else {
        GridD<float> g;
        grid_view(s, g);
        k_volume<float><<<512, 256, 0, s->stream>>>(g, s->ctl, s->rkf.k.A, vol);
    }
    CUDA_TRY(cudaGetLastError());
    s->launches += 1;
    double V = 0.0;
    CUDA_TRY(cudaMemcpyAsync(&V, vol, sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    const Ctl *c = (const Ctl *)s->ctl_host;
    memset(st, 0, sizeof(*st));
    st->t = c->t;
    st->dt_base = c->dt_base;
    st->step = c->step;
    st->done = c->done;
    st->V = V;
    st->V0 = s->V0;
    double a[4] = {0, 0, 0, 0};
    long long cap = 0;
    for (int k = 0; k < 4; k++)
        for (int j = 0; j < NSLOT; j++)
            a[k] += s->cfg.precision == FCAB_PREC_F32_ALL ? (double)c->accf[k][j] : c->accd[k][j];
    for (int j = 0; j < NSLOT; j++)
        cap += (long long)c->cap[j];
    st->V_rain = a[0];
    st->clamp_err = a[1];
    st->V_sea = a[2];
    st->V_bnd = a[3];
    st->V_in = c->V_in;
    st->cap_active = cap;
    st->cap_total = s->faces_per_step * (long long)(c->step - s->step0);
    st->dt_min_hits = c->dt_min_hits;
    st->dt_full_passes = c->full_passes;
    double den = st->V_rain + st->V_in + st->V0;
    if (den < 1e-30)
        den = 1e-30;
    st->E_mass = fabs(st->V + st->V_sea + st->V_bnd - st->V_rain - st->V_in - st->V0 -
                      st->clamp_err) /
                 den;
    s->h_cur_host = c->h_cur;
    return 0;
}

extern "C" int fcab_sim_download(FcabSim *s, void *h, void *hmax, void *tmax)
{
    CUDA_TRY(cudaMemcpyAsync(s->ctl_host, s->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    const Ctl *c = (const Ctl *)s->ctl_host;
    s->h_cur_host = c->h_cur;
    if (h)
        CUDA_TRY(get_field(s, h, c->h_cur ? s->h1 : s->h0, s->esize));
    if (hmax)
        CUDA_TRY(get_field(s, hmax, s->hmax, s->esize));
    if (tmax)
        CUDA_TRY(get_field(s, tmax, s->tmax, s->esize));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    return 0;
}

extern "C" int fcab_sim_layout(FcabSim *s, void **h, void **hmax, void **tmax, long long *pitch,
                               int *pad_rows, int *pad_cols)
{
    FcabPoll p;
    int rc = fcab_sim_poll(s, &p);
    if (rc)
        return rc;
    if (h)
        *h = s->h_cur_host ? s->h1 : s->h0;
    if (hmax)
        *hmax = s->hmax;
    if (tmax)
        *tmax = s->tmax;
    if (pitch)
        *pitch = s->pitch;
    if (pad_rows)
        *pad_rows = PADR;
    if (pad_cols)
        *pad_cols = PADC;
    return 0;
}

extern "C" long long fcab_sim_launches(FcabSim *s) { return s->launches; }

extern "C" int fcab_sim_info(FcabSim *s, FcabInfo *info)
{
    int rc = resolve_variant(s);
    if (rc)
        return rc;
    info->cols_per_lane = s->cpl;
    info->grid = s->grid;
    info->warps = s->warps_total;
    info->ctas_per_sm = s->occupancy;
    info->rain_field = s->rain_field ? 1 : 0;
    info->land_only = s->landonly ? 1 : 0;
    info->land_cells = s->land_cells;
    info->faces_per_step = s->faces_per_step;
    info->pitch = s->pitch;
    info->tma_rows = s->use_tma && s->L.tma_smem > 0 ? 1 : 0;
    return 0;
}

extern "C" int fcab_sim_set_config(FcabSim *s, const FcabConfig *cfg)
{
    const FcabConfig &o = s->cfg;
    if (cfg->nrows != o.nrows || cfg->ncols != o.ncols || cfg->precision != o.precision ||
        cfg->K != o.K)
        return fail(FCAB_ERR_ARG, "set_config cannot change the grid, precision or K");
    if (int rc = validate_config(cfg))
        return rc;
    const int keep_cpl = s->cpl;
    const int has_sea = s->esize == 8 ? s->rkd.has_sea : s->rkf.has_sea;
    const double cru = s->esize == 8 ? s->rkd.cr_uniform : (double)s->rkf.cr_uniform;
    const int inflow_ok = s->tc.inflow_ok;
    s->cfg = *cfg;
    if (s->esize == 8) {
        fill_runk<double>(s->rkd, *cfg, s->hn, s->hs);
        s->rkd.has_sea = has_sea;
        s->rkd.cr_uniform = cru;
    } else {
        fill_runk<float>(s->rkf, *cfg, s->hn, s->hs);
        s->rkf.has_sea = has_sea;
        s->rkf.cr_uniform = (float)cru;
    }
    const int p = cfg->precision;
    TimeCfg &tc = s->tc;
    tc.T_sim = as_real(cfg->T_sim, p);
    tc.out_every = as_real(cfg->out_every, p);
    tc.D_h = as_real(cfg->D_h, p);
    tc.phi = as_real(cfg->phi, p);
    tc.rain_end = cfg->rain_end;
    tc.inflow_peak = cfg->inflow_peak;
    tc.inflow_t_peak = cfg->inflow_t_peak;
    tc.inflow_t_end = cfg->inflow_t_end;
    tc.hyeto = cfg->hyeto;
    tc.max_steps = cfg->max_steps;
    tc.U = cfg->U > 0 ? cfg->U : 1;
    tc.inflow_ok = inflow_ok;
    tc.vseed_on = 1;
    tc.tail_vpass = 1;
    s->cpl = cfg->cols_per_lane ? pick_cpl(*cfg) : keep_cpl;
    s->variant_dirty = true;
    return 0;
}

extern "C" int fcab_sim_set_pause_every(FcabSim *s, int nsteps, int n_force_days)
{
    s->tc.progress_every = nsteps > 0 ? nsteps : 0;
    s->tc.n_force_days = n_force_days > 0 ? n_force_days : 0;
    if (s->graph) {
        cudaGraphExecDestroy(s->graph);   // kernel arguments changed
        s->graph = nullptr;
    }
    return 0;
}

extern "C" int fcab_sim_upload_state(FcabSim *s, const void *h, const void *hmax, const void *tmax)
{
    if (!s->uploaded)
        return fail(FCAB_ERR_STATE, "upload_state before upload");
    if (!h)
        return fail(FCAB_ERR_ARG, "h is required");
    s->h_cur_host = 0;
    CUDA_TRY(put_field(s, s->h0, h, s->esize, cudaMemcpyHostToDevice));
    CUDA_TRY(put_field(s, s->hmax, hmax ? hmax : h, s->esize, cudaMemcpyHostToDevice));
    if (tmax)
        CUDA_TRY(put_field(s, s->tmax, tmax, s->esize, cudaMemcpyHostToDevice));
    else
        CUDA_TRY(cudaMemsetAsync(s->tmax, 0, s->nelem * s->esize, s->stream));
    return 0;
}

// Adds hmax >= thr[j] on LAND cells into counts[j*N + a] (unpadded index),
// counts the flooded cells per threshold and the largest LAND hmax (at least
// 0), as FloodCA's k_ens_count does (src/cuda/kernels.cu:799-823).
template <typename T>
__global__ void k_count(GridD<T> g, int nthr, double t0, double t1, double t2, double t3,
                        uint16_t *counts, unsigned long long *flooded,
                        unsigned long long *maxbits)
{
    const double thr[4] = {t0, t1, t2, t3};
    unsigned long long f[4] = {0, 0, 0, 0};
    T mx = T(0);
    const long long N = (long long)g.nr * g.nc;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N;
         i += (long long)gridDim.x * blockDim.x) {
        const long long a = (i / g.nc + PADR) * g.pitch + i % g.nc + PADC;
        if (g.m[a] != M_LAND)
            continue;
        const T hm = g.hmax[a];
        if (hm > mx)
            mx = hm;
        for (int j = 0; j < nthr; j++) {
            if ((double)hm >= thr[j]) {
                if (counts)
                    counts[(long long)j * N + i]++;
                f[j]++;
            }
        }
    }
    for (int j = 0; j < 4; j++) {
        unsigned long long v = warp_sum(f[j]);
        if ((threadIdx.x & 31) == 0 && v)
            atomicAdd(&flooded[j], v);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const T vo = __shfl_xor_sync(0xffffffffu, mx, o);
        mx = vo > mx ? vo : mx;
    }
    if ((threadIdx.x & 31) == 0 && mx > T(0)) {
        const double d = (double)mx;
        atomicMax(maxbits, (unsigned long long)__double_as_longlong(d));
    }
}

extern "C" int fcab_sim_count_flooded(FcabSim *s, int nthr, const double *thr, uint16_t *counts,
                                      long long *flooded, double *max_depth)
{
    if (nthr < 1 || nthr > 4)
        return fail(FCAB_ERR_ARG, "%d thresholds, at most 4", nthr);
    double t[4] = {0, 0, 0, 0};
    for (int j = 0; j < nthr; j++)
        t[j] = thr[j];
    unsigned long long *d = (unsigned long long *)s->scratch;   // 4 counts + max
    CUDA_TRY(cudaMemsetAsync(d, 0, 5 * sizeof(unsigned long long), s->stream));
    if (s->esize == 8) {
        GridD<double> g;
        grid_view(s, g);
        k_count<double><<<1024, 256, 0, s->stream>>>(g, nthr, t[0], t[1], t[2], t[3], counts, d,
                                                    d + 4);
    } else {
        GridD<float> g;
        grid_view(s, g);
        k_count<float><<<1024, 256, 0, s->stream>>>(g, nthr, t[0], t[1], t[2], t[3], counts, d,
                                                   d + 4);
    }
    CUDA_TRY(cudaGetLastError());
    s->launches += 1;
    unsigned long long h[5];
    CUDA_TRY(cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    for (int j = 0; j < nthr; j++)
        flooded[j] = (long long)h[j];
    double mx;
    memcpy(&mx, &h[4], sizeof(double));
    *max_depth = mx;
    return 0;
}

extern "C" void *fcab_sim_stream(FcabSim *s) { return (void *)s->stream; }

// ---------------------------------------------------------------------------
// Slabs of a row-split domain.

static_assert(FCAB_SLAB_HALO < PADR, "halo rows live in the padding rows");

extern "C" int fcab_sim_set_slab(FcabSim *s, int halo_n, int halo_s)
{
    if (s->uploaded)
        return fail(FCAB_ERR_STATE, "set_slab after upload");
    if (halo_n < 0 || halo_n > FCAB_SLAB_HALO || halo_s < 0 || halo_s > FCAB_SLAB_HALO)
        return fail(FCAB_ERR_ARG, "halo rows %d / %d outside 0..%d", halo_n, halo_s,
                    FCAB_SLAB_HALO);
    s->slab = true;
    s->hn = halo_n;
    s->hs = halo_s;
    if (s->esize == 8)
        fill_runk<double>(s->rkd, s->cfg, s->hn, s->hs);
    else
        fill_runk<float>(s->rkf, s->cfg, s->hn, s->hs);
    // the seed and the deferral decision come from the reduced maximum, so
    // every slab defers alike; the driver then runs fcab_sim_slab_vfull
    s->tc.split = 1;
    s->variant_dirty = true;
    return 0;
}

extern "C" int fcab_sim_slab_step(FcabSim *s)
{
    if (!s->slab)
        return fail(FCAB_ERR_STATE, "slab_step on a session that is not a slab");
    if (!s->inited)
        return fail(FCAB_ERR_STATE, "slab_step before upload");
    int rc = resolve_variant(s);
    if (rc)
        return rc;
    if (s->esize == 8) {
        GridD<double> g;
        grid_view(s, g);
        CUDA_TRY(s->L.step(&g, &s->rkd, s->tc, s->ctl, s->warps_total, s->grid, s->stream,
                           step_smem(s)));
    } else {
        GridD<float> g;
        grid_view(s, g);
        CUDA_TRY(s->L.step(&g, &s->rkf, s->tc, s->ctl, s->warps_total, s->grid, s->stream,
                           step_smem(s)));
    }
    s->launches += 1;
    return 0;
}

extern "C" int fcab_sim_slab_vfull(FcabSim *s)
{
    if (!s->slab)
        return fail(FCAB_ERR_STATE, "slab_vfull on a session that is not a slab");
    if (!s->inited)
        return fail(FCAB_ERR_STATE, "slab_vfull before upload");
    int rc = resolve_variant(s);
    if (rc)
        return rc;
    const int full_grid = 2 * 148 * 4;
    if (s->esize == 8) {
        GridD<double> g;
        grid_view(s, g);
        CUDA_TRY(s->L.init(&g, &s->rkd, s->tc, s->ctl, full_grid, s->stream, 1));
    } else {
        GridD<float> g;
        grid_view(s, g);
        CUDA_TRY(s->L.init(&g, &s->rkf, s->tc, s->ctl, full_grid, s->stream, 1));
    }
    s->launches += 1;
    return 0;
}

extern "C" int fcab_sim_slab_vmax(FcabSim *s, unsigned long long **vmax)
{
    if (!s->slab)
        return fail(FCAB_ERR_STATE, "slab_vmax on a session that is not a slab");
    *vmax = &s->ctl->vmax_bits;
    return 0;
}

extern "C" int fcab_sim_slab_finalize(FcabSim *s)
{
    if (!s->slab)
        return fail(FCAB_ERR_STATE, "slab_finalize on a session that is not a slab");
    if (s->esize == 8)
        k_slab_finalize<double><<<1, 1, 0, s->stream>>>(s->rkd, s->tc, s->ctl);
    else
        k_slab_finalize<float><<<1, 1, 0, s->stream>>>(s->rkf, s->tc, s->ctl);
    CUDA_TRY(cudaGetLastError());
    s->launches += 1;
    return 0;
}

static int rows_copy(FcabSim *s, int row0, int nrows, void *buf, int to_buf)
{
    if (!s->uploaded)
        return fail(FCAB_ERR_STATE, "rows copy before upload");
    if (nrows < 0 || row0 < -s->hn || (long long)row0 + nrows > (long long)s->cfg.nrows + s->hs)
        return fail(FCAB_ERR_ARG, "rows [%d, %d) outside %d..%d", row0, row0 + nrows, -s->hn,
                    s->cfg.nrows + s->hs);
    if (nrows == 0)
        return 0;
    if (!buf)
        return fail(FCAB_ERR_ARG, "rows copy without a buffer");
    const long long N = (long long)nrows * s->cfg.ncols;
    const int blocks = (int)std::min<long long>((N + 255) / 256, 1024);
    if (s->esize == 8)
        k_rows_copy<double><<<blocks, 256, 0, s->stream>>>(s->ctl, (double *)s->h0,
                                                           (double *)s->h1, s->pitch, row0,
                                                           nrows, s->cfg.ncols, (double *)buf,
                                                           to_buf);
    else
        k_rows_copy<float><<<blocks, 256, 0, s->stream>>>(s->ctl, (float *)s->h0,
                                                          (float *)s->h1, s->pitch, row0, nrows,
                                                          s->cfg.ncols, (float *)buf, to_buf);
    CUDA_TRY(cudaGetLastError());
    s->launches += 1;
    return 0;
}

extern "C" int fcab_sim_rows_get(FcabSim *s, int row0, int nrows, void *dst)
{
    return rows_copy(s, row0, nrows, dst, 1);
}

extern "C" int fcab_sim_rows_put(FcabSim *s, int row0, int nrows, const void *src)
{
    return rows_copy(s, row0, nrows, const_cast<void *>(src), 0);
}

// Evaluates one device math helper over n inputs, for tests: which = 0
// RN(cbrt(x*x)) (exact mode), 1 min(x, RN(sqrt(g*y))) (exact mode), 2 the
// fast-mode cbrt(x*x) estimate.
__global__ void k_math_probe(int which, const float *x, const float *y, float *out, long long n,
                             float g)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        float r;
        if (which == 0)
            r = cbrt_sq_rn(x[i]);
        else if (which == 1)
            r = min_vcr_rn(x[i], g, y[i]);
        else if (which == 2)
            r = Mth<float, MATH_FAST>::cbrt_sq(x[i]);
        else if (which == 3)
            r = (__fsqrt_rn(x[i]) == sqrt_nr(x[i])) && (__frcp_rn(x[i]) == rcp_nr(x[i])) ? 1.f : 0.f;
        else if (which == 4)
            r = rcp_nr(x[i]);
        else if (which == 5)
            r = sqrt_nr(x[i]);
        else if (which == 6)
            r = div_mk(x[i], y[i], __frcp_rn(y[i]));
        else if (which == 7)
            r = __frcp_rn(x[i]);
        else if (which == 8)
            r = __fsqrt_rn(x[i]);
        else if (which == 10) {
            // the pair sweep's cube root: its value where it decides the
            // rounding itself, NaN where it defers to the exact evaluation
            bool u0, u1;
            const f2 c = cbrt_sq2(mk2(x[i], x[i]), u0, u1);
            r = u0 ? __int_as_float(0x7fc00000) : lo2(c);
        } else if (which == 11) {
            // the pair sweep's product then packed sum: two roundings,
            // RN(RN(x*y) + g)
            r = lo2(add2(mul2_sep(mk2(x[i], x[i]), mk2(y[i], y[i])), bc2(g)));
        } else
            r = __fdiv_rn(x[i], y[i]);
        out[i] = r;
    }
}

extern "C" int fcab_math_probe(int which, const float *x, const float *y, float *out, long long n,
                               float g)
{
    float *dx = nullptr, *dy = nullptr, *dout = nullptr;
    const size_t b = (size_t)n * sizeof(float);
    int rc = 0;
    if (cudaMalloc(&dx, b) != cudaSuccess || cudaMalloc(&dy, b) != cudaSuccess ||
        cudaMalloc(&dout, b) != cudaSuccess) {
        rc = fail(FCAB_ERR_CUDA, "math_probe alloc");
        goto done;
    }
    if (cudaMemcpy(dx, x, b, cudaMemcpyHostToDevice) != cudaSuccess ||
        (y && cudaMemcpy(dy, y, b, cudaMemcpyHostToDevice) != cudaSuccess)) {
        rc = fail(FCAB_ERR_CUDA, "math_probe copy");
        goto done;
    }
    k_math_probe<<<1024, 256>>>(which, dx, dy, dout, n, g);
    if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess ||
        cudaMemcpy(out, dout, b, cudaMemcpyDeviceToHost) != cudaSuccess)
        rc = fail(FCAB_ERR_CUDA, "math_probe run");
done:
    cudaFree(dx);
    cudaFree(dy);
    cudaFree(dout);
    return rc;
}

namespace fcab {

// Run constants of an FP32 configuration, for entry points that launch the
// step kernels without a session.
void make_run_params_f32(const FcabConfig &cfg, RunK<float> *rk, TimeCfg *tc)
{
    fill_runk<float>(*rk, cfg);
    memset(tc, 0, sizeof(*tc));
    const int p = cfg.precision;
    tc->T_sim = as_real(cfg.T_sim, p);
    tc->out_every = as_real(cfg.out_every, p);
    tc->D_h = as_real(cfg.D_h, p);
    tc->phi = as_real(cfg.phi, p);
    tc->rain_end = cfg.rain_end;
    tc->inflow_peak = cfg.inflow_peak;
    tc->inflow_t_peak = cfg.inflow_t_peak;
    tc->inflow_t_end = cfg.inflow_t_end;
    tc->hyeto = cfg.hyeto;
    tc->max_steps = cfg.max_steps;
    tc->U = cfg.U > 0 ? cfg.U : 1;
}

}  // namespace fcab
