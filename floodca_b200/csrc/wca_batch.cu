// Batched ensemble runs (fcab_batch_*): many sessions advanced together.
//
// Each member is an ordinary session (own padded grid, control block, dt,
// time, rain). A batched launch advances every active member by one step
// (k_step_batch); a CUDA graph of `graph_steps` launches is replayed until
// every member has reached the end of the current output window or of its
// run, then the next window opens (k_batch_window). The host reads one
// gathered activity flag per member between graph replays.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <vector>

#include "floodca_b200.h"
#include "wca_dispatch.h"
#include "wca_sim_internal.h"

using namespace fcab;

namespace {

__global__ void k_gather_active(const MemberD<float> *members, int n, int *flags)
{
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m < n) {
        const Ctl *c = members[m].ctl;
        flags[m] = c->active ? 1 : (c->done ? 0 : 2);   // 1 running, 2 paused, 0 done
    }
}

// The loop condition of a window graph: keep stepping while any member is
// active (running in the current window) and the pass count is below `cap`
// (a bound on one graph launch; the host launches the graph again if members
// are still running).
__global__ void k_batch_cond(const MemberD<float> *members, int n, cudaGraphConditionalHandle h,
                             unsigned long long *passes, unsigned long long cap)
{
    int any = 0;
    for (int m = threadIdx.x; m < n; m += blockDim.x)
        any |= members[m].ctl->active != 0;
    any = __syncthreads_or(any);
    if (threadIdx.x == 0) {
        const unsigned long long k = *passes + 1;
        *passes = k;
        cudaGraphSetConditional(h, any && k < cap ? 1u : 0u);
    }
}

int bfail(int code, const char *msg)
{
    set_error(msg);
    return code;
}

}  // namespace

struct FcabBatch {
    std::vector<FcabSim *> members;
    int n = 0;
    cudaStream_t stream = nullptr;
    VariantKey key{};
    BatchLaunchers L{};
    MemberD<float> *d_members = nullptr;
    int *d_unit_member = nullptr;
    int *d_need = nullptr;      // members whose step deferred its dt
    BatchQ *d_q = nullptr;
    int *d_flags = nullptr;
    int *h_flags = nullptr;     // pinned
    int total_units = 0, grid = 1, seg = 64;
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0;
    // one graph per output window: [open the window], then a conditional
    // while loop of `wsteps` steps per pass until no member is active
    cudaGraphExec_t wgraph = nullptr;
    int wsteps = 0;
    double wwindow = 0.0;
    bool wgraph_failed = false;     // conditional graphs unavailable: host-polled loop
    unsigned long long *d_passes = nullptr;
    long long launches = 0, windows = 0, replays = 0;
};

extern "C" int fcab_batch_create(FcabBatch **out, FcabSim *const *members, int n,
                                 int cols_per_lane, int seg_rows, const int *member_seg_rows,
                                 void *stream)
{
    *out = nullptr;
    if (n < 1 || !members)
        return bfail(FCAB_ERR_ARG, "fcab_batch_create: no members");
    FcabSim *m0 = members[0];
    for (int i = 0; i < n; i++) {
        const FcabSim *s = members[i];
        if (!s || !s->inited)
            return bfail(FCAB_ERR_STATE, "fcab_batch_create: member not uploaded");
        if (s->cfg.precision != FCAB_PREC_F32 || s->cfg.K != m0->cfg.K ||
            s->cfg.math != m0->cfg.math || s->landonly != m0->landonly ||
            s->rain_field != m0->rain_field || s->dev != m0->dev)
            return bfail(FCAB_ERR_ARG, "fcab_batch_create: members must share FP32 precision, K, "
                                       "math, rain form, mask form and device");
        if (s->tc.n_force_days > 0 || s->tc.progress_every > 0)
            return bfail(FCAB_ERR_ARG, "fcab_batch_create: members with forcing days or "
                                       "progress pauses run as single sessions");
        if (s->slab)
            return bfail(FCAB_ERR_ARG, "fcab_batch_create: a slab of a row-split domain "
                                       "steps through fcab_sim_slab_*");
    }
    FcabBatch *b = new FcabBatch();
    b->members.assign(members, members + n);
    b->n = n;
    b->stream = stream ? (cudaStream_t)stream : m0->stream;
    b->key.prec = FCAB_PREC_F32;
    b->key.K = m0->cfg.K;
    b->key.cpl = (cols_per_lane == 1 || cols_per_lane == 2 || cols_per_lane == 4) ? cols_per_lane : 2;
    if (b->key.K == 8 && b->key.cpl == 4)
        b->key.cpl = 2;
    b->key.math = m0->cfg.math;
    b->key.rainf = m0->rain_field ? 1 : 0;
    b->key.landonly = m0->landonly ? 1 : 0;
    // the pair sweep addresses the fields with 32-bit element offsets
    if (b->key.landonly && b->key.cpl == 2)
        for (int i = 0; i < n; i++) {
            const FcabSim *s = members[i];
            if ((long long)(s->cfg.nrows + s->hn + s->hs + 2 * PADR) * s->pitch >= (1ll << 31))
                b->key.cpl = 1;
        }
    if (!lookup_batch_f32(b->key, &b->L)) {
        delete b;
        return bfail(FCAB_ERR_ARG, "fcab_batch_create: no compiled batch variant");
    }
    b->seg = seg_rows > 0 ? seg_rows : 64;
    const int ow = 32 * b->key.cpl - 2 * (b->key.cpl == 1 ? 3 : 4);
    std::vector<MemberD<float>> md(n);
    std::vector<int> um;
    for (int i = 0; i < n; i++) {
        FcabSim *s = members[i];
        MemberD<float> &d = md[i];
        d.g.z = (const float *)s->z;
        d.g.n = (const float *)s->n;
        d.g.cr = s->rain_field ? (const float *)s->cr : nullptr;
        d.g.m = s->m;
        d.g.h0 = (float *)s->h0;
        d.g.h1 = (float *)s->h1;
        d.g.hmax = (float *)s->hmax;
        d.g.tmax = (float *)s->tmax;
        d.g.pitch = s->pitch;
        d.g.nr = s->cfg.nrows;
        d.g.nc = s->cfg.ncols;
        d.g.r_lo = 0;
        d.g.r_hi = s->cfg.nrows;
        d.rk = s->rkf;
        d.tc = s->tc;
        d.tc.vseed_on = 1;    // the graph runs the deferred full passes after each step
        d.ctl = s->ctl;
        d.strips = (s->cfg.ncols + ow - 1) / ow;
        d.seg = member_seg_rows && member_seg_rows[i] > 0 ? member_seg_rows[i] : b->seg;
        const int blocks = (s->cfg.nrows + d.seg - 1) / d.seg;
        d.units = d.strips * blocks;
        d.unit_off = (int)um.size();
        um.insert(um.end(), (size_t)d.units, i);
    }
    b->total_units = (int)um.size();
    cudaError_t e = cudaMalloc(&b->d_members, sizeof(MemberD<float>) * n);
    if (e == cudaSuccess)
        e = cudaMalloc(&b->d_unit_member, sizeof(int) * um.size());
    if (e == cudaSuccess)
        e = cudaMalloc(&b->d_need, sizeof(int) * n);
    if (e == cudaSuccess)
        e = cudaMalloc(&b->d_q, sizeof(BatchQ));
    if (e == cudaSuccess)
        e = cudaMalloc(&b->d_flags, sizeof(int) * n);
    if (e == cudaSuccess)
        e = cudaMallocHost(&b->h_flags, sizeof(int) * n);
    if (e == cudaSuccess)
        e = cudaMalloc(&b->d_passes, sizeof(unsigned long long));
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->d_members, md.data(), sizeof(MemberD<float>) * n,
                            cudaMemcpyHostToDevice, b->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->d_unit_member, um.data(), sizeof(int) * um.size(),
                            cudaMemcpyHostToDevice, b->stream);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(b->d_q, 0, sizeof(BatchQ), b->stream);
    int nsm = 1, per_sm = 1;
    if (e == cudaSuccess)
        e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, m0->dev);
    if (e == cudaSuccess)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, b->L.step_fn, 128, 0);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) {
        fcab_batch_destroy(b);
        return bfail(FCAB_ERR_CUDA, cudaGetErrorString(e));
    }
    b->grid = nsm * (per_sm > 0 ? per_sm : 1);
    *out = b;
    return 0;
}

extern "C" void fcab_batch_destroy(FcabBatch *b)
{
    if (!b)
        return;
    if (b->graph)
        cudaGraphExecDestroy(b->graph);
    if (b->wgraph)
        cudaGraphExecDestroy(b->wgraph);
    cudaFree(b->d_passes);
    cudaFree(b->d_members);
    cudaFree(b->d_unit_member);
    cudaFree(b->d_need);
    cudaFree(b->d_q);
    cudaFree(b->d_flags);
    if (b->h_flags)
        cudaFreeHost(b->h_flags);
    delete b;
}

static int batch_graph(FcabBatch *b, int steps)
{
    if (b->graph && b->graph_steps == steps)
        return 0;
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    cudaGraph_t g;
    cudaError_t e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess)
        return bfail(FCAB_ERR_CUDA, cudaGetErrorString(e));
    cudaError_t le = cudaSuccess;
    for (int i = 0; i < steps && le == cudaSuccess; i++) {
        le = b->L.step(b->d_members, b->d_unit_member, b->total_units, b->d_q, b->d_need,
                       b->grid, b->stream);
        if (le == cudaSuccess)
            le = b->L.vfull(b->d_members, b->d_need, b->d_q, 2 * 148 * 4, b->stream);
    }
    e = cudaStreamEndCapture(b->stream, &g);
    if (le != cudaSuccess || e != cudaSuccess)
        return bfail(FCAB_ERR_CUDA, "fcab_batch: graph capture failed");
    e = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess)
        return bfail(FCAB_ERR_CUDA, cudaGetErrorString(e));
    b->graph_steps = steps;
    return 0;
}

// Passes of the window loop in one graph launch at most (each `wsteps` steps).
constexpr unsigned long long WINDOW_PASS_CAP = 1ull << 20;

// One graph per output window: the window's opening (paced runs), then a
// conditional while node whose body is `steps` batch steps and the loop
// condition (k_batch_cond), so a window is one graph launch with no host
// round trip inside it. Returns nonzero (and leaves no graph) when the
// driver cannot build it.
static int window_graph(FcabBatch *b, int steps, double window_s)
{
    if (b->wgraph && b->wsteps == steps && b->wwindow == window_s)
        return 0;
    if (b->wgraph) {
        cudaGraphExecDestroy(b->wgraph);
        b->wgraph = nullptr;
    }
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaGraphCreate(&g, 0);
    cudaGraphConditionalHandle h = 0;
    if (e == cudaSuccess)
        e = cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault);
    // top level: reset the pass count, open the window
    if (e == cudaSuccess)
        e = cudaStreamBeginCaptureToGraph(b->stream, g, nullptr, nullptr, 0,
                                          cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        cudaError_t le = cudaMemsetAsync(b->d_passes, 0, sizeof(unsigned long long), b->stream);
        if (le == cudaSuccess && window_s > 0.0)
            le = b->L.window(b->d_members, b->n, window_s, b->stream);
        cudaGraph_t gc = nullptr;
        e = cudaStreamEndCapture(b->stream, &gc);
        if (e == cudaSuccess)
            e = le;
    }
    // the loop hangs off the last node of the top level
    std::vector<cudaGraphNode_t> leaves;
    if (e == cudaSuccess) {
        size_t nn = 0;
        e = cudaGraphGetNodes(g, nullptr, &nn);
        std::vector<cudaGraphNode_t> nodes(nn);
        if (e == cudaSuccess && nn)
            e = cudaGraphGetNodes(g, nodes.data(), &nn);
        for (size_t k = 0; k < nn && e == cudaSuccess; k++) {
            size_t nd = 0;
            e = cudaGraphNodeGetDependentNodes(nodes[k], nullptr, &nd);
            if (e == cudaSuccess && nd == 0)
                leaves.push_back(nodes[k]);
        }
    }
    // (the parameter struct has no default constructor: zeroed storage)
    alignas(cudaGraphNodeParams) unsigned char cpb[sizeof(cudaGraphNodeParams)];
    memset(cpb, 0, sizeof(cpb));
    cudaGraphNodeParams &cp = *reinterpret_cast<cudaGraphNodeParams *>(cpb);
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t cn = nullptr;
    if (e == cudaSuccess)
        e = cudaGraphAddNode(&cn, g, leaves.data(), leaves.size(), &cp);
    if (e == cudaSuccess) {
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        e = cudaStreamBeginCaptureToGraph(b->stream, body, nullptr, nullptr, 0,
                                          cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            cudaError_t le = cudaSuccess;
            for (int i = 0; i < steps && le == cudaSuccess; i++) {
                le = b->L.step(b->d_members, b->d_unit_member, b->total_units, b->d_q, b->d_need,
                               b->grid, b->stream);
                if (le == cudaSuccess)
                    le = b->L.vfull(b->d_members, b->d_need, b->d_q, 2 * 148 * 4, b->stream);
            }
            if (le == cudaSuccess) {
                k_batch_cond<<<1, 256, 0, b->stream>>>(b->d_members, b->n, h, b->d_passes,
                                                        WINDOW_PASS_CAP);
                le = cudaGetLastError();
            }
            cudaGraph_t bc = nullptr;
            e = cudaStreamEndCapture(b->stream, &bc);
            if (e == cudaSuccess)
                e = le;
        }
    }
    if (e == cudaSuccess)
        e = cudaGraphInstantiate(&b->wgraph, g, 0);
    if (g)
        cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        b->wgraph = nullptr;
        cudaGetLastError();     // clear the (non-sticky) error of the failed build
        return 1;
    }
    b->wsteps = steps;
    b->wwindow = window_s;
    return 0;
}

// Members running / paused at a window end, and the window loop's passes.
static int poll_members(FcabBatch *b, int *running, int *paused, unsigned long long *passes)
{
    k_gather_active<<<(b->n + 127) / 128, 128, 0, b->stream>>>(b->d_members, b->n, b->d_flags);
    b->launches += 1;
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->h_flags, b->d_flags, sizeof(int) * b->n, cudaMemcpyDeviceToHost,
                            b->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(passes, b->d_passes, sizeof(unsigned long long),
                            cudaMemcpyDeviceToHost, b->stream);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess)
        return bfail(FCAB_ERR_CUDA, cudaGetErrorString(e));
    *running = *paused = 0;
    for (int i = 0; i < b->n; i++) {
        *running += b->h_flags[i] == 1;
        *paused += b->h_flags[i] == 2;
    }
    return 0;
}

extern "C" int fcab_batch_run(FcabBatch *b, double window_s, int graph_steps, int max_windows)
{
    const bool paced = window_s > 0.0;
    const int steps = graph_steps > 0 ? graph_steps : 16;
    if (!b->wgraph_failed && window_graph(b, steps, paced ? window_s : 0.0) != 0)
        b->wgraph_failed = true;
    const bool wg = !b->wgraph_failed;
    cudaError_t e;
    int opened = 0;
    for (;;) {
        // the window: one graph launch, or its opening kernel before the
        // host-polled replays below
        if (wg) {
            e = cudaGraphLaunch(b->wgraph, b->stream);
            if (e != cudaSuccess)
                return bfail(FCAB_ERR_CUDA, cudaGetErrorString(e));
            b->replays += 1;
        } else if (paced) {
            e = b->L.window(b->d_members, b->n, window_s, b->stream);
            if (e != cudaSuccess)
                return bfail(FCAB_ERR_CUDA, cudaGetErrorString(e));
        }
        if (paced) {
            b->launches += 1;
            b->windows += 1;
            opened += 1;
        }
        int running = 0, paused = 0;
        unsigned long long passes = 0;
        int rc = poll_members(b, &running, &paused, &passes);
        if (rc)
            return rc;
        if (wg)
            b->launches += (long long)passes * (2 * steps + 1);
        // members still running: no window graph, or its pass cap was hit
        while (running) {
            rc = batch_graph(b, steps);
            if (rc)
                return rc;
            e = cudaGraphLaunch(b->graph, b->stream);
            if (e != cudaSuccess)
                return bfail(FCAB_ERR_CUDA, cudaGetErrorString(e));
            b->launches += 2 * steps;
            b->replays += 1;
            rc = poll_members(b, &running, &paused, &passes);
            if (rc)
                return rc;
        }
        if (!paused || !paced || (max_windows > 0 && opened >= max_windows))
            break;
    }
    return 0;
}

extern "C" int fcab_batch_info(FcabBatch *b, FcabBatchInfo *info)
{
    info->members = b->n;
    info->cols_per_lane = b->key.cpl;
    info->seg_rows = b->seg;
    info->grid = b->grid;
    info->total_units = b->total_units;
    info->launches = b->launches;
    info->windows = b->windows;
    info->graph_replays = b->replays;
    return 0;
}
