// Session state behind the opaque FcabSim handle.
#pragma once

#include <cuda_runtime.h>

#include "floodca_b200.h"
#include "wca_dispatch.h"

struct FcabSim {
    FcabConfig cfg;
    int dev = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    size_t esize = 4;            // element size of the state (4 or 8)
    long long pitch = 0;         // elements per padded row
    int rows_alloc = 0;
    size_t nelem = 0;            // elements per padded field
    void *z = nullptr, *n = nullptr, *cr = nullptr, *h0 = nullptr, *h1 = nullptr;
    void *hmax = nullptr, *tmax = nullptr;
    uint8_t *m = nullptr;
    void *tmpC = nullptr, *tmpR = nullptr;   // padded staging copies of C and Rday
    fcab::Ctl *ctl = nullptr;    // device control block
    void *ctl_host = nullptr;    // pinned mirror
    void *scratch = nullptr;     // 64 bytes of device scratch
    void *tmaps = nullptr;       // row-tile tensor maps of z, n, h0, h1 (device memory)
    bool use_tma = false;        // FP32 pair sweep rows by TMA
    fcab::RunK<float> rkf;
    fcab::RunK<double> rkd;
    fcab::TimeCfg tc;
    bool rain_field = false;
    bool landonly = false;       // mask-free kernel variant (all cells LAND)
    int cpl = 2, grid = 1, warps_total = 4, occupancy = 1;
    fcab::Launchers L;
    bool have_variant = false, variant_dirty = true;
    cudaGraphExec_t graph = nullptr;
    long long launches = 0;
    bool uploaded = false, inited = false;
    int h_cur_host = 0;
    int step0 = 0;
    double V0 = 0.0;
    long long land_cells = 0, open_faces = 0, faces_per_step = 0;
    // slab of a row-split domain: halo rows above (hn) and below (hs) the
    // session's own rows, carried by every uploaded array
    bool slab = false;
    int hn = 0, hs = 0;
};

namespace fcab {
// Records the calling thread's fcab_last_error() message (wca_sim.cu).
void set_error(const char *msg);
// Columns per lane of the step kernel for a configuration: cfg.cols_per_lane
// when set (1, 2 or 4), else by grid size (wca_sim.cu).
int pick_cpl(const FcabConfig &c);
// Warps of the step kernel's grid: enough to fill the resident slots (nsm SMs,
// per_sm CTAs of wpb warps) with segments of cfg.seg_rows rows when set,
// else an even split, at least 4 rows per warp (wca_sim.cu).
long long step_warps(const FcabConfig &c, int cpl, int nsm, int per_sm, int wpb);
// Run constants of an FP32 configuration (defined in wca_sim.cu).
void make_run_params_f32(const FcabConfig &cfg, RunK<float> *rk, TimeCfg *tc);
// Row-block copies between dense pageable host rows and pitched device rows
// through pinned staging buffers and several host threads (host_copy.cu).
// h2d_rows returns once the host rows have been read (the transfer may still
// run; later work on `stream` follows it); d2h_rows returns with the host
// rows written.
cudaError_t h2d_rows(void *dst, size_t dpitch, const void *src, size_t row_bytes, size_t rows,
                     cudaStream_t stream);
cudaError_t d2h_rows(void *dst, const void *src, size_t spitch, size_t row_bytes, size_t rows,
                     cudaStream_t stream);
// Caching allocator of session buffers (mem_cache.cu): freed blocks are kept
// per device for the next request of about the same size. A block must be
// idle (its stream synchronised) when it is freed.
cudaError_t cached_malloc(void **p, size_t bytes);
cudaError_t cached_malloc_host(void **p, size_t bytes);
void cached_free(void *p);
}  // namespace fcab
