// Caching allocator for session buffers. Freeing a session's device fields
// (hundreds of MB for a 4096^2 grid) with cudaFree took from 5 ms to almost
// 1 s on a B200, varying from call to call; a caller that runs one domain
// after another (fca_cuda_run per scenario, tests, benchmarks) would pay it
// every time. Freed blocks are kept per device and handed to the next
// request of the same size (up to 1/8 larger), up to a cap of cached bytes
// (FCAB_CACHE_BYTES, default a quarter of the device memory; 0 disables the
// cache). fcab_release_cached_memory() frees every cached block.
#include <cuda_runtime.h>

#include <cstdlib>
#include <map>
#include <mutex>
#include <unordered_map>

#include "wca_sim_internal.h"

namespace {

constexpr int MAX_DEV = 64;
constexpr int HOST = MAX_DEV;     // index of the pinned host cache

struct Cache {
    std::multimap<size_t, void *> idle;
    size_t idle_bytes = 0;
    size_t limit = 0;
    bool limit_set = false;
};

struct Live {
    size_t bytes;
    int where;      // device index, or HOST
};

std::mutex g_mu;
Cache g_cache[MAX_DEV + 1];
std::unordered_map<void *, Live> g_live;

size_t limit_of(Cache &c, int where)
{
    if (c.limit_set)
        return c.limit;
    c.limit_set = true;
    if (const char *e = getenv("FCAB_CACHE_BYTES")) {
        c.limit = (size_t)strtoull(e, nullptr, 10);
        return c.limit;
    }
    size_t fr = 0, tot = 0;
    if (where != HOST && cudaMemGetInfo(&fr, &tot) == cudaSuccess)
        c.limit = tot / 4;
    else
        c.limit = (size_t)256 << 20;
    return c.limit;
}

void *take(Cache &c, size_t bytes, size_t *got)
{
    auto it = c.idle.lower_bound(bytes);
    if (it == c.idle.end() || it->first > bytes + bytes / 8)
        return nullptr;
    void *p = it->second;
    *got = it->first;
    c.idle_bytes -= it->first;
    c.idle.erase(it);
    return p;
}

void release(Cache &c, int where)
{
    for (auto &kv : c.idle) {
        if (where == HOST)
            cudaFreeHost(kv.second);
        else
            cudaFree(kv.second);
    }
    c.idle.clear();
    c.idle_bytes = 0;
}

cudaError_t alloc(void **p, size_t bytes, int where)
{
    *p = nullptr;
    if (bytes == 0)
        bytes = 1;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        size_t got = 0;
        if (void *q = take(g_cache[where], bytes, &got)) {
            g_live[q] = Live{got, where};
            *p = q;
            return cudaSuccess;
        }
    }
    cudaError_t e = where == HOST ? cudaMallocHost(p, bytes) : cudaMalloc(p, bytes);
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        {
            std::lock_guard<std::mutex> lk(g_mu);
            release(g_cache[where], where);
        }
        e = where == HOST ? cudaMallocHost(p, bytes) : cudaMalloc(p, bytes);
    }
    if (e != cudaSuccess) {
        *p = nullptr;
        return e;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    g_live[*p] = Live{bytes, where};
    return cudaSuccess;
}

void dealloc(void *p)
{
    if (!p)
        return;
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_live.find(p);
    if (it == g_live.end())
        return;
    const Live l = it->second;
    g_live.erase(it);
    Cache &c = g_cache[l.where];
    if (c.idle_bytes + l.bytes > limit_of(c, l.where)) {
        if (l.where == HOST)
            cudaFreeHost(p);
        else
            cudaFree(p);
        return;
    }
    c.idle.emplace(l.bytes, p);
    c.idle_bytes += l.bytes;
}

}  // namespace

namespace fcab {

cudaError_t cached_malloc(void **p, size_t bytes)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return e;
    if (dev < 0 || dev >= MAX_DEV)
        return cudaMalloc(p, bytes);
    return alloc(p, bytes, dev);
}

cudaError_t cached_malloc_host(void **p, size_t bytes) { return alloc(p, bytes, HOST); }

void cached_free(void *p) { dealloc(p); }

}  // namespace fcab

extern "C" FCAB_API void fcab_release_cached_memory(void)
{
    std::lock_guard<std::mutex> lk(g_mu);
    for (int w = 0; w <= MAX_DEV; w++)
        release(g_cache[w], w);
}
