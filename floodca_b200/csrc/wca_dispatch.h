// Kernel variant table shared by the session code and the per-precision
// instantiation units (wca_inst_*.cu), so the variants compile in parallel.
#pragma once

#include <cuda_runtime.h>

#include "wca_kernels.cuh"

namespace fcab {

// Selects one compiled step-kernel variant.
struct VariantKey {
    int prec;   // FCAB_PREC_*
    int K;      // 4 or 8
    int cpl;    // 1, 2 or 4
    int math;   // MATH_*
    int rainf;  // per-cell rain field
    int landonly; // every cell LAND (mask not read, padding at PAD_Z)
};

// Type-erased launchers; `g`, `rk` point at GridD<T>/RunK<T> of the variant's T.
struct Launchers {
    cudaError_t (*step)(const void *g, const void *rk, const TimeCfg &tc, Ctl *ctl,
                        int warps_total, int grid, cudaStream_t s, int smem);
    // full velocity pass + step control: the first step's dt, or
    // (only_if_needed) a dt deferred by a step whose pruned maximum fell
    // below its seed
    cudaError_t (*init)(const void *g, const void *rk, const TimeCfg &tc, Ctl *ctl, int grid,
                        cudaStream_t s, int only_if_needed);
    const void *step_fn;   // __global__ symbol, for occupancy queries
    int threads;           // threads per CTA of the step kernel
    int tma_smem;          // dynamic shared memory of its TMA row source (0: none)
};

// Batched-ensemble launchers (FP32 state, FP64 accumulation).
struct BatchLaunchers {
    cudaError_t (*step)(const void *members, const int *unit_member, int total_units, BatchQ *q,
                        int *need_list, int grid, cudaStream_t s);
    // full velocity pass of the members whose step deferred its dt
    cudaError_t (*vfull)(const void *members, const int *need_list, BatchQ *q, int grid,
                         cudaStream_t s);
    cudaError_t (*window)(const void *members, int n, double window, cudaStream_t s);
    const void *step_fn;
};
bool lookup_batch_f32(const VariantKey &k, BatchLaunchers *out);

template <typename T, typename AccT, int K, int CPL, int MATH, bool RAINF, bool LAND>
cudaError_t launch_batch(const void *members, const int *unit_member, int total_units, BatchQ *q,
                         int *need_list, int grid, cudaStream_t s)
{
    k_step_batch<T, AccT, K, CPL, MATH, RAINF, LAND><<<grid, 128, 0, s>>>(
        static_cast<const MemberD<T> *>(members), unit_member, total_units, q, need_list);
    return cudaGetLastError();
}

template <typename T, int K, int MATH>
cudaError_t launch_batch_vfull(const void *members, const int *need_list, BatchQ *q, int grid,
                               cudaStream_t s)
{
    k_batch_vfull<T, K, MATH><<<grid, 256, 0, s>>>(static_cast<const MemberD<T> *>(members),
                                                  need_list, q);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_window(const void *members, int n, double window, cudaStream_t s)
{
    k_batch_window<T><<<(n + 127) / 128, 128, 0, s>>>(static_cast<const MemberD<T> *>(members),
                                                       n, window);
    return cudaGetLastError();
}

// Returns false when the variant is not compiled.
bool lookup_f32(const VariantKey &k, Launchers *out);
bool lookup_f32all(const VariantKey &k, Launchers *out);
bool lookup_f64(const VariantKey &k, Launchers *out);

template <typename T, typename AccT, int K, int CPL, int MATH, bool RAINF, bool LAND>
cudaError_t launch_step(const void *g, const void *rk, const TimeCfg &tc, Ctl *ctl,
                        int warps_total, int grid, cudaStream_t s, int smem)
{
    k_step<T, AccT, K, CPL, MATH, RAINF, LAND><<<grid, step_threads<CPL, MATH>(), smem, s>>>(
        *static_cast<const GridD<T> *>(g), *static_cast<const RunK<T> *>(rk), tc, ctl,
        warps_total);
    return cudaGetLastError();
}

template <typename T, int K, int MATH>
cudaError_t launch_init(const void *g, const void *rk, const TimeCfg &tc, Ctl *ctl, int grid,
                        cudaStream_t s, int only_if_needed)
{
    k_init_dt<T, K, MATH><<<grid, 256, 0, s>>>(*static_cast<const GridD<T> *>(g),
                                              *static_cast<const RunK<T> *>(rk), tc, ctl,
                                              only_if_needed);
    return cudaGetLastError();
}

template <typename T, typename AccT, int K, int CPL, int MATH, bool RAINF, bool LAND>
Launchers make_launchers()
{
    Launchers L;
    L.step = &launch_step<T, AccT, K, CPL, MATH, RAINF, LAND>;
    L.init = &launch_init<T, K, MATH>;
    L.step_fn = (const void *)&k_step<T, AccT, K, CPL, MATH, RAINF, LAND>;
    L.threads = step_threads<CPL, MATH>();
    L.tma_smem = use_pair_sweep<T, K, CPL, LAND>() ? tma_smem_bytes(L.threads / 32) : 0;
    return L;
}

// Expands the (K, CPL, RAINF) combinations for one (T, AccT, MATH).
template <typename T, typename AccT, int MATH>
bool lookup_kcr(const VariantKey &k, Launchers *out)
{
#define FCAB_CASE(KK, CC, RR)                                                    \
    if (k.K == KK && k.cpl == CC && (k.rainf != 0) == RR) {                      \
        *out = k.landonly ? make_launchers<T, AccT, KK, CC, MATH, RR, true>()   \
                          : make_launchers<T, AccT, KK, CC, MATH, RR, false>(); \
        return true;                                                             \
    }
    FCAB_CASE(4, 1, false) FCAB_CASE(4, 1, true)
    FCAB_CASE(4, 2, false) FCAB_CASE(4, 2, true)
    FCAB_CASE(4, 4, false) FCAB_CASE(4, 4, true)
    FCAB_CASE(8, 1, false) FCAB_CASE(8, 1, true)
    FCAB_CASE(8, 2, false) FCAB_CASE(8, 2, true)
    FCAB_CASE(8, 4, false) FCAB_CASE(8, 4, true)
#undef FCAB_CASE
    return false;
}

}  // namespace fcab
