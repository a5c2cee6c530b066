// Host <-> device copies of row blocks between pageable host arrays and the
// padded device fields, through pinned staging buffers filled and drained by
// several host threads at once. A pageable cudaMemcpy runs at the speed of
// one driver staging thread; here each worker thread owns two pinned slots
// and its own stream, so host memcpy, PCIe transfer and the other workers
// overlap.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "wca_sim_internal.h"

namespace {

constexpr int MAX_DEV = 16;
constexpr int MAX_WORKERS = 16;
constexpr size_t SLOT = 4u << 20;    // bytes per pinned slot

struct Worker {
    cudaStream_t st = nullptr;
    char *slot[2] = {nullptr, nullptr};
    cudaEvent_t ev[2] = {nullptr, nullptr};
    cudaEvent_t done = nullptr;
};

struct Pool {
    bool ready = false;
    int n = 0;
    Worker w[MAX_WORKERS];
    cudaEvent_t start = nullptr;
};

std::mutex g_mu;
Pool g_pool[MAX_DEV];

int workers_wanted()
{
    if (const char *e = getenv("FCAB_COPY_THREADS")) {
        const int v = atoi(e);
        if (v >= 1)
            return std::min(v, MAX_WORKERS);
    }
    const unsigned hc = std::thread::hardware_concurrency();
    return (int)std::max(1u, std::min(4u, hc / 2));
}

cudaError_t ensure(Pool &p)
{
    if (p.ready)
        return cudaSuccess;
    // resources made by an earlier, failed attempt are kept and not remade
    cudaError_t e;
    p.n = workers_wanted();
    if (!p.start && (e = cudaEventCreateWithFlags(&p.start, cudaEventDisableTiming)) != cudaSuccess)
        return e;
    for (int i = 0; i < p.n; i++) {
        Worker &w = p.w[i];
        if (!w.st && (e = cudaStreamCreateWithFlags(&w.st, cudaStreamNonBlocking)) != cudaSuccess)
            return e;
        if (!w.done && (e = cudaEventCreateWithFlags(&w.done, cudaEventDisableTiming)) != cudaSuccess)
            return e;
        for (int k = 0; k < 2; k++) {
            if (!w.slot[k] && (e = cudaMallocHost(&w.slot[k], SLOT)) != cudaSuccess)
                return e;
            if (!w.ev[k] && (e = cudaEventCreateWithFlags(&w.ev[k], cudaEventDisableTiming)) != cudaSuccess)
                return e;
        }
    }
    p.ready = true;
    return cudaSuccess;
}

struct Job {
    char *dev;          // device rows, pitch dpitch
    size_t dpitch;
    char *host;         // dense host rows
    size_t row_bytes, rows, rows_per_chunk, nchunks;
};

// Worker t copies chunks t, t + n, ... host -> device.
cudaError_t h2d_worker(Worker &w, const Job &j, int t, int n)
{
    cudaError_t e = cudaSuccess;
    int k = 0;
    for (size_t c = (size_t)t; c < j.nchunks && e == cudaSuccess; c += (size_t)n, k ^= 1) {
        const size_t r0 = c * j.rows_per_chunk;
        const size_t nr = std::min(j.rows_per_chunk, j.rows - r0);
        if ((e = cudaEventSynchronize(w.ev[k])) != cudaSuccess)   // the slot's last copy
            break;
        memcpy(w.slot[k], j.host + r0 * j.row_bytes, nr * j.row_bytes);
        e = cudaMemcpy2DAsync(j.dev + r0 * j.dpitch, j.dpitch, w.slot[k], j.row_bytes,
                              j.row_bytes, nr, cudaMemcpyHostToDevice, w.st);
        if (e == cudaSuccess)
            e = cudaEventRecord(w.ev[k], w.st);
    }
    return e;
}

// Worker t copies chunks t, t + n, ... device -> host, one copy in flight
// while the previous slot drains.
cudaError_t d2h_worker(Worker &w, const Job &j, int t, int n)
{
    cudaError_t e = cudaSuccess;
    size_t pend = (size_t)-1;   // chunk in flight in slot k ^ 1
    int k = 0;
    auto drain = [&](size_t c, int slot) -> cudaError_t {
        const size_t r0 = c * j.rows_per_chunk;
        const size_t nr = std::min(j.rows_per_chunk, j.rows - r0);
        cudaError_t ee = cudaEventSynchronize(w.ev[slot]);
        if (ee == cudaSuccess)
            memcpy(j.host + r0 * j.row_bytes, w.slot[slot], nr * j.row_bytes);
        return ee;
    };
    for (size_t c = (size_t)t; c < j.nchunks && e == cudaSuccess; c += (size_t)n) {
        const size_t r0 = c * j.rows_per_chunk;
        const size_t nr = std::min(j.rows_per_chunk, j.rows - r0);
        e = cudaMemcpy2DAsync(w.slot[k], j.row_bytes, j.dev + r0 * j.dpitch, j.dpitch,
                              j.row_bytes, nr, cudaMemcpyDeviceToHost, w.st);
        if (e == cudaSuccess)
            e = cudaEventRecord(w.ev[k], w.st);
        if (e == cudaSuccess && pend != (size_t)-1)
            e = drain(pend, k ^ 1);
        pend = c;
        k ^= 1;
    }
    if (e == cudaSuccess && pend != (size_t)-1)
        e = drain(pend, k ^ 1);
    return e;
}

cudaError_t run_job(Job j, cudaStream_t stream, bool to_device)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return e;
    if (j.rows == 0 || j.row_bytes == 0)
        return cudaSuccess;
    if (dev < 0 || dev >= MAX_DEV || j.row_bytes > SLOT) {
        // rows wider than a slot: one pageable copy
        if (to_device)
            return cudaMemcpy2DAsync(j.dev, j.dpitch, j.host, j.row_bytes, j.row_bytes, j.rows,
                                     cudaMemcpyHostToDevice, stream);
        e = cudaMemcpy2DAsync(j.host, j.row_bytes, j.dev, j.dpitch, j.row_bytes, j.rows,
                              cudaMemcpyDeviceToHost, stream);
        return e == cudaSuccess ? cudaStreamSynchronize(stream) : e;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    Pool &p = g_pool[dev];
    if ((e = ensure(p)) != cudaSuccess)
        return e;
    j.rows_per_chunk = std::max<size_t>(1, SLOT / j.row_bytes);
    j.nchunks = (j.rows + j.rows_per_chunk - 1) / j.rows_per_chunk;
    const int n = (int)std::min<size_t>((size_t)p.n, j.nchunks);
    // the copies follow the work already queued on `stream`
    if ((e = cudaEventRecord(p.start, stream)) != cudaSuccess)
        return e;
    for (int t = 0; t < n; t++)
        if ((e = cudaStreamWaitEvent(p.w[t].st, p.start, 0)) != cudaSuccess)
            return e;
    std::vector<cudaError_t> errs((size_t)n, cudaSuccess);
    std::vector<std::thread> th;
    auto body = [&](int t) {
        cudaSetDevice(dev);
        errs[(size_t)t] = to_device ? h2d_worker(p.w[t], j, t, n) : d2h_worker(p.w[t], j, t, n);
    };
    for (int t = 1; t < n; t++)
        th.emplace_back(body, t);
    body(0);
    for (auto &x : th)
        x.join();
    for (int t = 0; t < n; t++)
        if (errs[(size_t)t] != cudaSuccess)
            return errs[(size_t)t];
    // later work on `stream` follows the copies
    for (int t = 0; t < n; t++) {
        if ((e = cudaEventRecord(p.w[t].done, p.w[t].st)) != cudaSuccess ||
            (e = cudaStreamWaitEvent(stream, p.w[t].done, 0)) != cudaSuccess)
            return e;
    }
    return cudaSuccess;
}

}  // namespace

namespace fcab {

cudaError_t h2d_rows(void *dst, size_t dpitch, const void *src, size_t row_bytes, size_t rows,
                     cudaStream_t stream)
{
    Job j{(char *)dst, dpitch, (char *)const_cast<void *>(src), row_bytes, rows, 0, 0};
    return run_job(j, stream, true);
}

cudaError_t d2h_rows(void *dst, const void *src, size_t spitch, size_t row_bytes, size_t rows,
                     cudaStream_t stream)
{
    Job j{(char *)const_cast<void *>(src), spitch, (char *)dst, row_bytes, rows, 0, 0};
    return run_job(j, stream, false);
}

}  // namespace fcab
