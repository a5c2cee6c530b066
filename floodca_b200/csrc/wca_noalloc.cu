// fcab_run_noalloc: the fused WCA step for callers that cannot allocate
// device memory.
//
// Who needs it: a host process whose device memory belongs to another
// allocator (a framework's caching pool, an arena sized at start-up) or a
// pipeline that must not call cudaMalloc/cudaFree once running, because
// those calls synchronise the whole device and can stall every other stream
// of the process. The session API (fcab_sim_create) allocates its working
// fields per grid, so such callers could not use it.
//
// How: the step kernel's working memory (padded copies of the fields, the
// ping-pong depth buffer, the control block) lives in one file-scope
// __device__ array of NOALLOC_MAX_PADDED padded cells, about 15 MB, which
// every GPU that loads the library holds until the process exits. The caller
// passes device arrays for the inputs and outputs. Nothing here allocates.
//
// Host code must not use g_noalloc_scratch as a device address (it is a
// host-side stand-in for the symbol); the address comes from
// cudaGetSymbolAddress, looked up once per device on that device's first call.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <mutex>

#include "floodca_b200.h"
#include "wca_dispatch.h"
#include "wca_sim_internal.h"

using namespace fcab;

namespace {

// Capacity in padded cells: (nrows + 16) * round_up(ncols + 132, 32) must not
// exceed it (a 512 x 768 grid fits, as does any grid of up to ~390k cells).
constexpr long long NOALLOC_MAX_PADDED = 1ll << 19;
constexpr size_t CTL_BYTES = (sizeof(Ctl) + 255) / 256 * 256;
constexpr size_t FIELD_BYTES = (size_t)NOALLOC_MAX_PADDED * sizeof(float);
// Ctl | 7 float fields (z, n, h0, h1, hmax, tmax, cr) | mask | 256 B misc
constexpr size_t SCRATCH_BYTES = CTL_BYTES + 7 * FIELD_BYTES + NOALLOC_MAX_PADDED + 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[SCRATCH_BYTES];

constexpr int MAX_DEVICES = 64;
std::mutex g_mu;
unsigned char *g_base[MAX_DEVICES];

thread_local char g_msg[256];

int noalloc_fail(int code, const char *msg)
{
    snprintf(g_msg, sizeof(g_msg), "fcab_run_noalloc: %s", msg);
    set_error(g_msg);
    return code;
}

// Device address of the scratch array on the current device.
int scratch_base(unsigned char **out)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES)
        return noalloc_fail(FCAB_ERR_CUDA, "no current device");
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_base[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return noalloc_fail(FCAB_ERR_CUDA, cudaGetErrorString(e));
        g_base[dev] = static_cast<unsigned char *>(p);
    }
    *out = g_base[dev];
    return 0;
}

// Copies the caller's row-major fields into the padded scratch fields
// (padding was cleared by the caller of this kernel).
struct PackDst {
    float *z, *n, *h0, *hmax, *tmax, *cr;
    uint8_t *m;
    long long pitch;
    int nr, nc;
};

__global__ void k_pack(const float *z, const float *n, const float *C, const float *R,
                       const uint8_t *mask, const float *h, const float *hmax,
                       const float *tmax, PackDst d)
{
    const long long N = (long long)d.nr * d.nc;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N;
         i += (long long)gridDim.x * blockDim.x) {
        const long long a = (i / d.nc + PADR) * d.pitch + i % d.nc + PADC;
        d.z[a] = z[i];
        d.n[a] = n[i];
        d.m[a] = mask[i];
        d.h0[a] = h[i];
        d.hmax[a] = hmax[i];
        d.tmax[a] = tmax ? tmax[i] : 0.0f;
        d.cr[a] = (C && R) ? C[i] * R[i] : 0.0f;
    }
}

__global__ void k_unpack(GridD<float> g, const Ctl *ctl, float *h, float *hmax, float *tmax)
{
    const float *hc = ctl->h_cur ? g.h1 : g.h0;
    const long long N = (long long)g.nr * g.nc;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N;
         i += (long long)gridDim.x * blockDim.x) {
        const long long a = (i / g.nc + PADR) * g.pitch + i % g.nc + PADC;
        h[i] = hc[a];
        hmax[i] = g.hmax[a];
        if (tmax)
            tmax[i] = g.tmax[a];
    }
}

// Starts the control block; the inflow cell is checked here, on the device
// (a cell that is not LAND receives no inflow volume), so the call never
// waits for the stream.
__global__ void k_ctl_start(Ctl *c, const uint8_t *mask, long long inflow_cell)
{
    c->t = 0.0;
    c->step = 0;
    c->dt_base = 0.0;
    c->force_day = -1;
    c->h_cur = 0;
    c->inflow_off = inflow_cell >= 0 && mask[inflow_cell] != M_LAND;
}

// Open faces per step: one per LAND cell on each open edge
// (FloodCA src/common/model.c:442-479), summed into *count.
__global__ void k_count_open(const uint8_t *mask, int nr, int nc, int en, int es, int ew, int ee,
                             unsigned long long *count)
{
    unsigned long long n = 0;
    const long long N = (long long)nr * nc;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N;
         i += (long long)gridDim.x * blockDim.x) {
        if (mask[i] != M_LAND)
            continue;
        const int r = (int)(i / nc), c = (int)(i % nc);
        n += (r == 0 && en) + (r == nr - 1 && es) + (c == 0 && ew) + (c == nc - 1 && ee);
    }
    n = warp_sum(n);
    if ((threadIdx.x & 31) == 0 && n)
        atomicAdd(count, n);
}

}  // namespace

extern "C" int fcab_run_noalloc(const FcabConfig *cfg, const float *z, const float *n,
                                const float *C, const float *Rday, const uint8_t *mask,
                                float *h, float *hmax, float *tmax, void *stream,
                                FcabStats *stats)
{
    if (!cfg || !z || !n || !mask || !h || !hmax)
        return noalloc_fail(FCAB_ERR_ARG, "cfg, z, n, mask, h and hmax are required");
    if (h == hmax || (tmax && (tmax == h || tmax == hmax)))
        return noalloc_fail(FCAB_ERR_ARG, "h, hmax and tmax must be distinct arrays");
    if (cfg->precision != FCAB_PREC_F32)
        return noalloc_fail(FCAB_ERR_ARG, "only the FP32 precision (FCAB_PREC_F32) is available");
    if (cfg->max_steps <= 0)
        return noalloc_fail(FCAB_ERR_ARG, "max_steps must be > 0 (a fixed number of steps)");
    if (cfg->K != 4 && cfg->K != 8)
        return noalloc_fail(FCAB_ERR_ARG, "K must be 4 or 8");
    if (cfg->nrows < 1 || cfg->ncols < 1)
        return noalloc_fail(FCAB_ERR_ARG, "empty grid");
    const long long pitch = ((long long)PADC + cfg->ncols + 128 + 31) / 32 * 32;
    const long long nelem = pitch * ((long long)cfg->nrows + 2 * PADR);
    if (nelem > NOALLOC_MAX_PADDED) {
        char m[160];
        snprintf(m, sizeof(m), "grid %dx%d needs %lld padded cells, limit %lld", cfg->nrows,
                 cfg->ncols, nelem, NOALLOC_MAX_PADDED);
        return noalloc_fail(FCAB_ERR_ARG, m);
    }
    unsigned char *base = nullptr;
    int rc = scratch_base(&base);
    if (rc)
        return rc;
    cudaStream_t s = (cudaStream_t)stream;

    Ctl *ctl = reinterpret_cast<Ctl *>(base);
    float *f = reinterpret_cast<float *>(base + CTL_BYTES);
    GridD<float> g;
    float *fz = f, *fn = f + nelem, *fh0 = f + 2 * nelem, *fh1 = f + 3 * nelem;
    float *fhm = f + 4 * nelem, *ftm = f + 5 * nelem, *fcr = f + 6 * nelem;
    uint8_t *fm = reinterpret_cast<uint8_t *>(f + 7 * nelem);
    // misc: V0, V, open faces per step
    double *vol = reinterpret_cast<double *>(base + CTL_BYTES + 7 * FIELD_BYTES +
                                             NOALLOC_MAX_PADDED);
    unsigned long long *nopen = reinterpret_cast<unsigned long long *>(vol + 2);
    g.z = fz;
    g.n = fn;
    g.cr = fcr;
    g.m = fm;
    g.h0 = fh0;
    g.h1 = fh1;
    g.hmax = fhm;
    g.tmax = ftm;
    g.pitch = pitch;
    g.nr = cfg->nrows;
    g.nc = cfg->ncols;
    g.r_lo = 0;
    g.r_hi = cfg->nrows;

    // The array keeps the previous call's contents: clear everything that
    // must start at zero (control block, padding, accumulators).
#define NA_TRY(x)                                                                \
    do {                                                                         \
        cudaError_t e_ = (x);                                                    \
        if (e_ != cudaSuccess)                                                   \
            return noalloc_fail(FCAB_ERR_CUDA, cudaGetErrorString(e_));          \
    } while (0)
    NA_TRY(cudaMemsetAsync(ctl, 0, sizeof(Ctl), s));
    NA_TRY(cudaMemsetAsync(f, 0, 7 * (size_t)nelem * sizeof(float), s));
    NA_TRY(cudaMemsetAsync(fm, M_WALL, (size_t)nelem, s));
    NA_TRY(cudaMemsetAsync(vol, 0, 256, s));
    PackDst pd{fz, fn, fh0, fhm, ftm, fcr, fm, pitch, cfg->nrows, cfg->ncols};
    k_pack<<<512, 256, 0, s>>>(z, n, C, Rday, mask, h, hmax, tmax, pd);
    NA_TRY(cudaGetLastError());
    const bool inflow_set =
        cfg->inflow_cell >= 0 && cfg->inflow_cell < (long long)cfg->nrows * cfg->ncols;
    k_ctl_start<<<1, 1, 0, s>>>(ctl, mask, inflow_set ? cfg->inflow_cell : -1);
    NA_TRY(cudaGetLastError());
    if (stats && cfg->boundary == FCA_BND_OPEN) {
        k_count_open<<<128, 256, 0, s>>>(mask, cfg->nrows, cfg->ncols, cfg->edge_n, cfg->edge_s,
                                         cfg->edge_w, cfg->edge_e, nopen);
        NA_TRY(cudaGetLastError());
    }

    RunK<float> rk;
    TimeCfg tc;
    make_run_params_f32(*cfg, &rk, &tc);
    rk.has_sea = 1;          // the generic kernel tests SEA neighbours itself
    rk.cr_uniform = 0.0f;
    tc.inflow_ok = inflow_set ? 1 : 0;      // k_ctl_start drops it for a non-LAND cell

    VariantKey key;
    key.prec = FCAB_PREC_F32;
    key.K = cfg->K;
    key.cpl = pick_cpl(*cfg);
    key.math = cfg->math == FCAB_MATH_FAST ? MATH_FAST : MATH_EXACT;
    key.rainf = 1;
    key.landonly = 0;
    Launchers L;
    if (!lookup_f32(key, &L))
        return noalloc_fail(FCAB_ERR_ARG, "no compiled kernel variant");
    int dev = 0, nsm = 1, per_sm = 1;
    NA_TRY(cudaGetDevice(&dev));
    NA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    NA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, L.step_fn, L.threads, 0));
    const int wpb = L.threads / 32;
    const int grid = (int)((step_warps(*cfg, key.cpl, nsm, per_sm, wpb) + wpb - 1) / wpb);

    if (stats) {   // V0, the LAND volume of the initial depth
        k_volume<float><<<256, 256, 0, s>>>(g, ctl, rk.k.A, vol);
        NA_TRY(cudaGetLastError());
    }
    NA_TRY(L.init(&g, &rk, tc, ctl, nsm * 4, s, 0));
    for (int k = 0; k < cfg->max_steps; k++)
        NA_TRY(L.step(&g, &rk, tc, ctl, grid * wpb, grid, s, 0));
    k_unpack<<<512, 256, 0, s>>>(g, ctl, h, hmax, tmax);
    NA_TRY(cudaGetLastError());

    if (stats) {
        k_volume<float><<<256, 256, 0, s>>>(g, ctl, rk.k.A, vol + 1);
        NA_TRY(cudaGetLastError());
        Ctl hc;
        double V[2] = {0.0, 0.0};
        unsigned long long nop = 0;
        NA_TRY(cudaMemcpyAsync(&hc, ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s));
        NA_TRY(cudaMemcpyAsync(V, vol, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
        NA_TRY(cudaMemcpyAsync(&nop, nopen, sizeof(nop), cudaMemcpyDeviceToHost, s));
        NA_TRY(cudaStreamSynchronize(s));
        memset(stats, 0, sizeof(*stats));
        stats->t = hc.t;
        stats->dt_base = hc.dt_base;
        stats->step = hc.step;
        stats->done = hc.done;
        stats->V0 = V[0];
        stats->V = V[1];
        for (int j = 0; j < NSLOT; j++) {
            stats->V_rain += hc.accd[0][j];
            stats->clamp_err += hc.accd[1][j];
            stats->V_sea += hc.accd[2][j];
            stats->V_bnd += hc.accd[3][j];
            stats->cap_active += (long long)hc.cap[j];
        }
        stats->V_in = hc.V_in;
        stats->dt_min_hits = hc.dt_min_hits;
        stats->dt_full_passes = hc.full_passes;
        // every face counts once per step (src/common/model.c:394-487)
        const long long nr = cfg->nrows, nc = cfg->ncols;
        const long long faces = nr * (nc - 1) + (nr - 1) * nc +
                                (cfg->K == 8 ? 2 * (nr - 1) * (nc - 1) : 0) + (long long)nop;
        stats->cap_total = faces * (long long)hc.step;
        double den = stats->V_rain + stats->V_in + stats->V0;
        den = den < 1e-30 ? 1e-30 : den;
        const double num = stats->V + stats->V_sea + stats->V_bnd - stats->V_rain -
                           stats->V_in - stats->V0 - stats->clamp_err;
        stats->E_mass = (num < 0 ? -num : num) / den;
    }
#undef NA_TRY
    return 0;
}
