// Layers of the flood-depth surrogate (a 4-level U-Net, BF16 weights and
// activations, FP32 accumulation) for sm_100a.
//
// Activation layout: NHWC bf16 with a one-pixel zero border, [N][H+2][W+2][C]
// (C a multiple of 16). Seen as a [P][C] matrix (P = N*(H+2)*(W+2)), the 3x3
// tap (ky, kx) of output pixel p reads input pixel p + (ky-1)*(W+2) + (kx-1),
// so a convolution is a GEMM whose A rows are shifted rows of one matrix:
// no im2col buffer, and TMA fills rows outside [0, P) with zeros. Border
// pixels of every activation and gradient buffer stay zero (kernels never
// write them), which is the convolution's zero padding.
//
// Tensor-core kernels (tcgen05, operands staged by TMA, accumulator in TMEM):
//   k_conv_gemm   forward conv (bias, ReLU) and the data gradient (the
//                 forward kernel on dY with the flipped, transposed weights)
//   k_conv_wgrad  weight gradient, split over pixels, FP32 atomics
// Weights: [Cout][9][Cin] (tap = ky*3 + kx).
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cstdint>
#include <cstdio>
#include <mutex>

#include "floodca_b200.h"
#include "wca_sim_internal.h"

namespace unet {

typedef __nv_bfloat16 bf16;

// ---------------------------------------------------------------------------
// PTX wrappers

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for the phase with the given parity; gives up after about 2 s.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity)
{
    const long long t0 = clock64();
    while (!mbar_try(bar, parity)) {
        if (clock64() - t0 > (1ll << 32))
            return false;
    }
    return true;
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *map, uint32_t bar,
                                            int c0, int c1)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%3, %4}], [%2];" ::"r"(dst),
        "l"((uint64_t)map), "r"(bar), "r"(c0), "r"(c1)
        : "memory");
}

__device__ __forceinline__ void tmem_alloc(uint32_t dst_smem, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst_smem),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
                 : "memory");
}

__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }

// D[tmem] (+)= A * B^T, bf16 operands from shared-memory descriptors, FP32 D.
__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                          uint32_t idesc, uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// Arrives on the mbarrier once every MMA issued so far by this thread is done.
__device__ __forceinline__ void umma_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

// 32 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32])
{
    uint32_t r[32];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; i++)
        v[i] = __uint_as_float(r[i]);
}

// Shared-memory matrix descriptor (sm_100 format): start address, leading and
// stride byte offsets (16-byte units), version 1, swizzle layout type.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo,
                                              uint32_t layout)
{
    uint64_t d = (uint64_t)((saddr & 0x3FFFFu) >> 4);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)layout << 61;
    return d;
}

// Instruction descriptor of kind::f16: BF16 A and B, FP32 D, M x N.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, bool a_mn, bool b_mn)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16) |
           ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// Swizzle of a K-major tile whose rows are CK bf16 (2*CK bytes).
template <int CK>
struct KSw {
    static constexpr uint32_t layout = CK == 64 ? 2u : CK == 32 ? 4u : 6u;  // 128B / 64B / 32B
    static constexpr uint32_t sbo = 8u * 2u * CK;                           // 8-row atom bytes
};

__device__ int g_err;   // first error code seen by a kernel of this file (0: none)

__device__ __forceinline__ void set_err(int code) { atomicCAS(&g_err, 0, code); }

__device__ __forceinline__ bool interior(int p, int P, int Hp, int Wp)
{
    if (p >= P)
        return false;
    const int q = p % (Hp * Wp);
    const int yy = q / Wp, xx = q - yy * Wp;
    return yy >= 1 && yy <= Hp - 2 && xx >= 1 && xx <= Wp - 2;
}

// ---------------------------------------------------------------------------
// Implicit-GEMM 3x3 convolution: M = 128 pixels per CTA, N = BN output
// channels, K = 9 taps x Cin in chunks of CK channels.
// Warp 0 lane 0 issues TMA loads, warp 1 lane 0 issues MMAs; all four warps
// run the epilogue (TMEM lane quarter of warp w = tile rows 32w..32w+31).

struct GemmArgs {
    int P, Hp, Wp;     // padded pixel count, padded height and width
    int Cin;           // channels of the A matrix
    int Cout;          // channels (row width) of the output matrix
    const float *bias; // [Cout] or null
    bf16 *y;           // [P][Cout]
    int relu;
};

template <int CK, int BN>
struct GemmCfg {
    static constexpr int A_BYTES = 128 * CK * 2;
    static constexpr int B_BYTES = BN * CK * 2;
    static constexpr int TX_BYTES = A_BYTES + B_BYTES;              // bytes of the two boxes
    static constexpr int STAGE = (TX_BYTES + 1023) / 1024 * 1024;   // 1024-aligned stage stride
    static constexpr int STAGES = (196608 / STAGE) < 8 ? (196608 / STAGE) : 8;
    static constexpr uint32_t TCOLS = BN <= 32 ? 32 : BN <= 64 ? 64 : BN <= 128 ? 128 : 256;
    static constexpr int SMEM = 1024 + STAGES * STAGE + (2 * STAGES + 1) * 8 + 16;
};

template <int CK, int BN>
__global__ void __launch_bounds__(128, 1)
k_conv_gemm(const __grid_constant__ CUtensorMap tx, const __grid_constant__ CUtensorMap tw, GemmArgs a)
{
    using Cfg = GemmCfg<CK, BN>;
    constexpr int S = Cfg::STAGES;
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    uint8_t *sm = smem_raw + (base - raw);
    const uint32_t bar0 = base + S * Cfg::STAGE;   // full[S], empty[S], done
    uint32_t *tslot = (uint32_t *)(sm + S * Cfg::STAGE + (2 * S + 1) * 8);
    auto full = [&](int s) { return bar0 + 8u * s; };
    auto empty = [&](int s) { return bar0 + 8u * (S + s); };
    const uint32_t done = bar0 + 8u * (2 * S);
    auto sA = [&](int s) { return base + (uint32_t)(s * Cfg::STAGE); };
    auto sB = [&](int s) { return base + (uint32_t)(s * Cfg::STAGE + Cfg::A_BYTES); };

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int p0 = blockIdx.x * 128;
    const int co0 = blockIdx.y * BN;
    if (threadIdx.x == 0) {
        for (int s = 0; s < S; s++) {
            mbar_init(full(s), 1);
            mbar_init(empty(s), 1);
        }
        mbar_init(done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 0)
        tmem_alloc(smem_u32(tslot), Cfg::TCOLS);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    const int cpt = a.Cin / CK;
    const int nk = 9 * cpt;

    if (warp == 0 && lane == 0) {
        for (int kb = 0; kb < nk; kb++) {
            const int s = kb % S;
            if (kb >= S && !mbar_wait(empty(s), (uint32_t)((kb / S) - 1) & 1u)) {
                set_err(1);
                break;
            }
            const int tap = kb / cpt, c0 = (kb - tap * cpt) * CK;
            const int shift = (tap / 3 - 1) * a.Wp + (tap % 3 - 1);
            mbar_expect_tx(full(s), (uint32_t)Cfg::TX_BYTES);
            tma_load_2d(sA(s), &tx, full(s), c0, p0 + shift);
            tma_load_2d(sB(s), &tw, full(s), tap * a.Cin + c0, co0);
        }
    } else if (warp == 1 && lane == 0) {
        constexpr uint32_t idesc = idesc_bf16(128, BN, false, false);
        for (int kb = 0; kb < nk; kb++) {
            const int s = kb % S;
            if (!mbar_wait(full(s), (uint32_t)(kb / S) & 1u)) {
                set_err(2);
                break;
            }
            tc_fence_after();
#pragma unroll
            for (int kk = 0; kk < CK / 16; kk++) {
                const uint64_t ad = smem_desc(sA(s) + 32u * kk, 16u, KSw<CK>::sbo, KSw<CK>::layout);
                const uint64_t bd = smem_desc(sB(s) + 32u * kk, 16u, KSw<CK>::sbo, KSw<CK>::layout);
                umma_bf16(tmem, ad, bd, idesc, (kb | kk) != 0 ? 1u : 0u);
            }
            umma_commit(empty(s));
        }
        umma_commit(done);
    }
    __syncwarp();
    if (!mbar_wait(done, 0))
        set_err(3);
    __syncwarp();
    tc_fence_after();

    const int row = warp * 32 + lane;
    const int p = p0 + row;
    const bool store = interior(p, a.P, a.Hp, a.Wp);
#pragma unroll 1
    for (int c = 0; c < BN; c += 32) {
        float v[32];
        tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
        if (store && co0 + c < a.Cout) {
            __align__(16) bf16 o[32];
#pragma unroll
            for (int j = 0; j < 32; j++) {
                float x = v[j];
                if (a.bias)
                    x += a.bias[co0 + c + j];
                if (a.relu)
                    x = fmaxf(x, 0.0f);
                o[j] = __float2bfloat16_rn(x);
            }
            uint4 *dst = (uint4 *)(a.y + (size_t)p * a.Cout + co0 + c);
            const uint4 *src = (const uint4 *)o;
#pragma unroll
            for (int j = 0; j < 4; j++)
                dst[j] = src[j];
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
        tmem_dealloc(tmem, Cfg::TCOLS);
}

// ---------------------------------------------------------------------------
// Weight gradient: dW[co][tap][ci] += sum_p dY[p][co] * X[p + shift(tap)][ci]
// as M = 128 output channels x N = 64*NB input channels x K = pixels, both
// operands MN-major (channels contiguous): each is loaded as boxes of 64
// channels x 64 pixels (128-byte swizzle; K groups of 8 pixels 1024 B apart,
// 64-channel blocks 8 KB apart). Each CTA takes one tap, one channel tile and
// one pixel range and adds its partial sums with FP32 atomics.

struct WgArgs {
    int P, Wp, Cin, Cout;
    int kpc;      // 64-pixel steps per CTA
    float *dw;    // [Cout][9][Cin]
};

template <int NB>
struct WgCfg {
    static constexpr int A_BYTES = 2 * 8192;
    static constexpr int B_BYTES = NB * 8192;
    static constexpr int STAGE = A_BYTES + B_BYTES;
    static constexpr int STAGES = 4;
    static constexpr uint32_t TCOLS = NB == 1 ? 64 : NB == 2 ? 128 : 256;
    static constexpr int SMEM = 1024 + STAGES * STAGE + (2 * STAGES + 1) * 8 + 16;
};

template <int NB>
__global__ void __launch_bounds__(128, 1)
k_conv_wgrad(const __grid_constant__ CUtensorMap tdy, const __grid_constant__ CUtensorMap tx, WgArgs a)
{
    using Cfg = WgCfg<NB>;
    constexpr int S = Cfg::STAGES;
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    uint8_t *sm = smem_raw + (base - raw);
    const uint32_t bar0 = base + S * Cfg::STAGE;
    uint32_t *tslot = (uint32_t *)(sm + S * Cfg::STAGE + (2 * S + 1) * 8);
    auto full = [&](int s) { return bar0 + 8u * s; };
    auto empty = [&](int s) { return bar0 + 8u * (S + s); };
    const uint32_t done = bar0 + 8u * (2 * S);
    auto sA = [&](int s) { return base + (uint32_t)(s * Cfg::STAGE); };
    auto sB = [&](int s) { return base + (uint32_t)(s * Cfg::STAGE + Cfg::A_BYTES); };

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tap = blockIdx.y % 9;
    const int co0 = (blockIdx.y / 9) * 128;
    const int ci0 = blockIdx.z * 64 * NB;
    const int kb0 = blockIdx.x * a.kpc;
    const int ksteps_total = (a.P + 63) / 64;
    int nk = ksteps_total - kb0;
    nk = nk < a.kpc ? nk : a.kpc;
    if (nk <= 0)
        return;     // uniform across the CTA, before any allocation
    const int na = (a.Cout - co0) >= 128 ? 2 : ((a.Cout - co0) + 63) / 64;
    int nb = (a.Cin - ci0 + 63) / 64;
    nb = nb < NB ? nb : NB;
    const int shift = (tap / 3 - 1) * a.Wp + (tap % 3 - 1);

    if (threadIdx.x == 0) {
        for (int s = 0; s < S; s++) {
            mbar_init(full(s), 1);
            mbar_init(empty(s), 1);
        }
        mbar_init(done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 0)
        tmem_alloc(smem_u32(tslot), Cfg::TCOLS);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;

    if (warp == 0 && lane == 0) {
        for (int k = 0; k < nk; k++) {
            const int s = k % S;
            if (k >= S && !mbar_wait(empty(s), (uint32_t)((k / S) - 1) & 1u)) {
                set_err(4);
                break;
            }
            const int px = (kb0 + k) * 64;
            mbar_expect_tx(full(s), (uint32_t)(na + nb) * 8192u);
            for (int j = 0; j < na; j++)
                tma_load_2d(sA(s) + 8192u * j, &tdy, full(s), co0 + 64 * j, px);
            for (int j = 0; j < nb; j++)
                tma_load_2d(sB(s) + 8192u * j, &tx, full(s), ci0 + 64 * j, px + shift);
        }
    } else if (warp == 1 && lane == 0) {
        // N = 64 * nb columns (the blocks that were loaded)
        const uint32_t idesc = idesc_bf16(128, 64 * nb, true, true);
        for (int k = 0; k < nk; k++) {
            const int s = k % S;
            if (!mbar_wait(full(s), (uint32_t)(k / S) & 1u)) {
                set_err(5);
                break;
            }
            tc_fence_after();
#pragma unroll
            for (int kk = 0; kk < 4; kk++) {
                const uint64_t ad = smem_desc(sA(s) + 2048u * kk, 8192u, 1024u, 2u);
                const uint64_t bd = smem_desc(sB(s) + 2048u * kk, 8192u, 1024u, 2u);
                umma_bf16(tmem, ad, bd, idesc, (k | kk) != 0 ? 1u : 0u);
            }
            umma_commit(empty(s));
        }
        umma_commit(done);
    }
    __syncwarp();
    if (!mbar_wait(done, 0))
        set_err(6);
    __syncwarp();
    tc_fence_after();

    const int co = co0 + warp * 32 + lane;
    const bool live = co < a.Cout;
#pragma unroll 1
    for (int c = 0; c < 64 * nb; c += 32) {
        float v[32];
        tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
        if (live) {
            float *dst = a.dw + ((size_t)co * 9 + tap) * a.Cin + ci0 + c;
#pragma unroll
            for (int j = 0; j < 32; j++)
                if (ci0 + c + j < a.Cin)
                    atomicAdd(dst + j, v[j]);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
        tmem_dealloc(tmem, Cfg::TCOLS);
}

// ---------------------------------------------------------------------------
// The other layers (CUDA cores; each is bandwidth-bound). Pixel (n, y, x) of
// an (H, W) image is row (n*(H+2) + y+1)*(W+2) + x+1 of its matrix.

__device__ __forceinline__ long long prow(int n, int y, int x, int H, int W)
{
    return ((long long)n * (H + 2) + y + 1) * (W + 2) + x + 1;
}

// 2x2 max pooling; idx keeps the arg max (0..3) for the backward pass.
__global__ void k_maxpool2(const bf16 *x, bf16 *y, uint8_t *idx, int N, int H, int W, int C)
{
    const int Ho = H / 2, Wo = W / 2;
    const long long total = (long long)N * Ho * Wo * C;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(i % C);
        long long t = i / C;
        const int ox = (int)(t % Wo);
        t /= Wo;
        const int oy = (int)(t % Ho);
        const int n = (int)(t / Ho);
        float best = -INFINITY;
        int bi = 0;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const float v = __bfloat162float(x[prow(n, 2 * oy + (k >> 1), 2 * ox + (k & 1), H, W) * C + c]);
            if (v > best) {
                best = v;
                bi = k;
            }
        }
        y[prow(n, oy, ox, Ho, Wo) * C + c] = __float2bfloat16_rn(best);
        idx[i] = (uint8_t)bi;
    }
}

__global__ void k_maxpool2_bwd(const bf16 *dy, const uint8_t *idx, bf16 *dx, int N, int H, int W, int C)
{
    const int Ho = H / 2, Wo = W / 2;
    const long long total = (long long)N * Ho * Wo * C;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(i % C);
        long long t = i / C;
        const int ox = (int)(t % Wo);
        t /= Wo;
        const int oy = (int)(t % Ho);
        const int n = (int)(t / Ho);
        const bf16 g = dy[prow(n, oy, ox, Ho, Wo) * C + c];
        const int bi = idx[i];
        const bf16 z = __float2bfloat16_rn(0.0f);
#pragma unroll
        for (int k = 0; k < 4; k++)
            dx[prow(n, 2 * oy + (k >> 1), 2 * ox + (k & 1), H, W) * C + c] = k == bi ? g : z;
    }
}

// Nearest-neighbour 2x upsampling of an (H, W) image to (2H, 2W).
__global__ void k_upsample2(const bf16 *x, bf16 *y, int N, int H, int W, int C)
{
    const int Ho = 2 * H, Wo = 2 * W;
    const long long total = (long long)N * Ho * Wo * C;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(i % C);
        long long t = i / C;
        const int ox = (int)(t % Wo);
        t /= Wo;
        const int oy = (int)(t % Ho);
        const int n = (int)(t / Ho);
        y[prow(n, oy, ox, Ho, Wo) * C + c] = x[prow(n, oy >> 1, ox >> 1, H, W) * C + c];
    }
}

// Gradient of the upsampling: each (H, W) pixel sums its four children.
__global__ void k_upsample2_bwd(const bf16 *dy, bf16 *dx, int N, int H, int W, int C)
{
    const long long total = (long long)N * H * W * C;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(i % C);
        long long t = i / C;
        const int x = (int)(t % W);
        t /= W;
        const int y = (int)(t % H);
        const int n = (int)(t / H);
        float s = 0.0f;
#pragma unroll
        for (int k = 0; k < 4; k++)
            s += __bfloat162float(dy[prow(n, 2 * y + (k >> 1), 2 * x + (k & 1), 2 * H, 2 * W) * C + c]);
        dx[prow(n, y, x, H, W) * C + c] = __float2bfloat16_rn(s);
    }
}

// Channel concatenation [a | b] over the interior pixels (and its split).
__global__ void k_concat(const bf16 *a, int Ca, const bf16 *b, int Cb, bf16 *y, int N, int H, int W,
                         int backward)
{
    const int C = Ca + Cb;
    const long long total = (long long)N * H * W * C;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(i % C);
        long long t = i / C;
        const int x = (int)(t % W);
        t /= W;
        const int yy = (int)(t % H);
        const int n = (int)(t / H);
        const long long r = prow(n, yy, x, H, W);
        if (!backward) {
            y[r * C + c] = c < Ca ? a[r * Ca + c] : b[r * Cb + (c - Ca)];
        } else {
            if (c < Ca)
                ((bf16 *)a)[r * Ca + c] = y[r * C + c];
            else
                ((bf16 *)b)[r * Cb + (c - Ca)] = y[r * C + c];
        }
    }
}

// y += x (bf16, FP32 sum).
__global__ void k_add(bf16 *y, const bf16 *x, long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        y[i] = __float2bfloat16_rn(__bfloat162float(y[i]) + __bfloat162float(x[i]));
}

// g *= (y > 0) over the whole matrix (borders are zero in g).
__global__ void k_relu_bwd(bf16 *g, const bf16 *y, long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        if (!(__bfloat162float(y[i]) > 0.0f))
            g[i] = __float2bfloat16_rn(0.0f);
    }
}

__device__ __forceinline__ uint32_t hash32(uint32_t x)
{
    x ^= x >> 16;
    x *= 0x7feb352dU;
    x ^= x >> 15;
    x *= 0x846ca68bU;
    x ^= x >> 16;
    return x;
}

// Inverted dropout in place: keep with probability 1-p, scale kept by
// 1/(1-p). The mask is a hash of (seed, element), so the backward pass
// regenerates it. Border pixels stay zero.
__global__ void k_dropout(bf16 *x, long long n, float p, uint32_t seed)
{
    const uint32_t thr = (uint32_t)(p * 4294967296.0);
    const float scale = 1.0f / (1.0f - p);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const uint32_t h = hash32((uint32_t)i ^ hash32(seed + (uint32_t)(i >> 32) * 0x9e3779b9U));
        const float v = __bfloat162float(x[i]);
        x[i] = __float2bfloat16_rn(h >= thr ? v * scale : 0.0f);
    }
}

// db[c] += sum over pixels of g[p][c].
__global__ void k_bias_grad(const bf16 *g, long long P, int C, float *db)
{
    const int c = threadIdx.x % C;
    const int lanes = blockDim.x / C;
    const int sub = threadIdx.x / C;
    if (sub >= lanes)
        return;
    float s = 0.0f;
    for (long long p = (long long)blockIdx.x * lanes + sub; p < P; p += (long long)gridDim.x * lanes)
        s += __bfloat162float(g[p * C + c]);
    atomicAdd(db + c, s);
}

// Output head: 1x1 convolution C -> 1, FP32 result on the unpadded grid.
__global__ void k_head_fwd(const bf16 *x, const float *w, const float *b, float *out, int N, int H,
                           int W, int C)
{
    const long long total = (long long)N * H * W;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int xx = (int)(i % W);
        const long long t = i / W;
        const int yy = (int)(t % H);
        const int n = (int)(t / H);
        const bf16 *r = x + prow(n, yy, xx, H, W) * C;
        float s = b[0];
        for (int c = 0; c < C; c++)
            s += w[c] * __bfloat162float(r[c]);
        out[i] = s;
    }
}

// Mean squared error of the head against the target, and its gradients:
// dx (bf16, padded), dw[c], db (accumulated), loss (accumulated sum).
__global__ void k_head_bwd(const bf16 *x, const float *w, const float *out, const float *target,
                           bf16 *dx, float *dw, float *db, float *loss, int N, int H, int W, int C,
                           float inv_count)
{
    __shared__ float s_dw[256];
    __shared__ float s_db, s_loss;
    for (int c = threadIdx.x; c < C; c += blockDim.x)
        s_dw[c] = 0.0f;
    if (threadIdx.x == 0)
        s_db = s_loss = 0.0f;
    __syncthreads();
    const long long total = (long long)N * H * W;
    float ldb = 0.0f, lloss = 0.0f;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int xx = (int)(i % W);
        const long long t = i / W;
        const int yy = (int)(t % H);
        const int n = (int)(t / H);
        const long long r = prow(n, yy, xx, H, W) * C;
        const float e = out[i] - target[i];
        lloss += e * e;
        const float d = 2.0f * e * inv_count;
        ldb += d;
        for (int c = 0; c < C; c++) {
            dx[r + c] = __float2bfloat16_rn(d * w[c]);
            atomicAdd(&s_dw[c], d * __bfloat162float(x[r + c]));
        }
    }
    atomicAdd(&s_db, ldb);
    atomicAdd(&s_loss, lloss);
    __syncthreads();
    for (int c = threadIdx.x; c < C; c += blockDim.x)
        atomicAdd(dw + c, s_dw[c]);
    if (threadIdx.x == 0) {
        atomicAdd(db, s_db);
        atomicAdd(loss, s_loss);
    }
}

// Master FP32 weights [Cout][9][Cin] -> bf16 copy (forward) and the bf16
// weights of the data gradient, wt[ci][tap][co] = w[co][8 - tap][ci].
__global__ void k_prep_weights(const float *w, bf16 *wb, bf16 *wt, int Cout, int Cin)
{
    const long long total = (long long)Cout * 9 * Cin;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int ci = (int)(i % Cin);
        const long long t = i / Cin;
        const int tap = (int)(t % 9);
        const int co = (int)(t / 9);
        const bf16 v = __float2bfloat16_rn(w[i]);
        wb[i] = v;
        wt[((long long)ci * 9 + (8 - tap)) * Cout + co] = v;
    }
}

// Adam with bias correction (c1 = 1 - beta1^t, c2 = 1 - beta2^t).
__global__ void k_adam(float *w, const float *g, float *m, float *v, long long n, float lr, float b1,
                       float b2, float eps, float c1, float c2, float wd)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i] + wd * w[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

// FP32 inputs [N][H][W][Cs] -> bf16 padded matrix with C >= Cs channels.
__global__ void k_pack_input(const float *in, int Cs, bf16 *x, int C, int N, int H, int W)
{
    const long long total = (long long)N * H * W * C;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(i % C);
        const long long t = i / C;
        const int xx = (int)(t % W);
        const long long t2 = t / W;
        const int yy = (int)(t2 % H);
        const int n = (int)(t2 / H);
        const float v = c < Cs ? in[t * Cs + c] : 0.0f;
        x[prow(n, yy, xx, H, W) * C + c] = __float2bfloat16_rn(v);
    }
}

// ---------------------------------------------------------------------------
// Host side

int fail(int code, const char *msg)
{
    fcab::set_error(msg);
    return code;
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
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

// 2D bf16 map over a row-major [rows][cols] matrix, box (bc, br).
bool make_map(CUtensorMap *m, const void *ptr, long long rows, int cols, int bc, int br,
              CUtensorMapSwizzle sw)
{
    auto fn = encode_fn();
    if (!fn || ((uintptr_t)ptr & 15) || (cols * 2) % 16)
        return false;
    cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)cols * 2};
    cuuint32_t box[2] = {(cuuint32_t)bc, (cuuint32_t)br};
    cuuint32_t es[2] = {1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, (void *)ptr, dims, strides, box, es,
              CU_TENSOR_MAP_INTERLEAVE_NONE, sw, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int CK, int BN>
cudaError_t launch_gemm(const CUtensorMap &tx, const CUtensorMap &tw, const GemmArgs &a, int n_tiles,
                        cudaStream_t st)
{
    using Cfg = GemmCfg<CK, BN>;
    static bool attr_set[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (!attr_set[dev & 63]) {
        cudaError_t e = cudaFuncSetAttribute(k_conv_gemm<CK, BN>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, Cfg::SMEM);
        if (e != cudaSuccess)
            return e;
        attr_set[dev & 63] = true;
    }
    dim3 grid((unsigned)((a.P + 127) / 128), (unsigned)n_tiles);
    k_conv_gemm<CK, BN><<<grid, 128, Cfg::SMEM, st>>>(tx, tw, a);
    return cudaGetLastError();
}

template <int CK>
cudaError_t gemm_bn(const CUtensorMap &tx, const CUtensorMap &tw, const GemmArgs &a, int bn,
                    int n_tiles, cudaStream_t st)
{
    switch (bn) {
    case 32: return launch_gemm<CK, 32>(tx, tw, a, n_tiles, st);
    case 64: return launch_gemm<CK, 64>(tx, tw, a, n_tiles, st);
    case 96: return launch_gemm<CK, 96>(tx, tw, a, n_tiles, st);
    case 128: return launch_gemm<CK, 128>(tx, tw, a, n_tiles, st);
    case 192: return launch_gemm<CK, 192>(tx, tw, a, n_tiles, st);
    case 256: return launch_gemm<CK, 256>(tx, tw, a, n_tiles, st);
    default: return cudaErrorInvalidValue;
    }
}

// y[P][Cout] = conv3x3(x[P][Cin], w[Cout][9][Cin]) (+ bias, ReLU).
int conv_gemm(const void *x, int N, int H, int W, int Cin, const void *w, int Cout,
              const float *bias, int relu, void *y, cudaStream_t st)
{
    if (N < 1 || H < 1 || W < 1 || Cin % 16 || Cout % 32 || Cout < 32)
        return fail(FCAB_ERR_ARG, "conv: Cin must be a multiple of 16 and Cout of 32");
    const int CK = Cin % 64 == 0 ? 64 : Cin % 32 == 0 ? 32 : 16;
    int bn = Cout;
    while (bn > 256)
        bn /= 2;
    if (Cout % bn || bn % 32)
        return fail(FCAB_ERR_ARG, "conv: unsupported Cout");
    const long long P = (long long)N * (H + 2) * (W + 2);
    if (P >= (1ll << 31) - 256)
        return fail(FCAB_ERR_ARG, "conv: too many pixels");
    const CUtensorMapSwizzle sw = CK == 64 ? CU_TENSOR_MAP_SWIZZLE_128B
                                  : CK == 32 ? CU_TENSOR_MAP_SWIZZLE_64B
                                             : CU_TENSOR_MAP_SWIZZLE_32B;
    CUtensorMap tx, tw;
    if (!make_map(&tx, x, P, Cin, CK, 128, sw) || !make_map(&tw, w, Cout, 9 * Cin, CK, bn, sw))
        return fail(FCAB_ERR_CUDA, "conv: tensor map encoding failed");
    GemmArgs a;
    a.P = (int)P;
    a.Hp = H + 2;
    a.Wp = W + 2;
    a.Cin = Cin;
    a.Cout = Cout;
    a.bias = bias;
    a.y = (bf16 *)y;
    a.relu = relu;
    cudaError_t e = CK == 64 ? gemm_bn<64>(tx, tw, a, bn, Cout / bn, st)
                    : CK == 32 ? gemm_bn<32>(tx, tw, a, bn, Cout / bn, st)
                               : gemm_bn<16>(tx, tw, a, bn, Cout / bn, st);
    if (e != cudaSuccess)
        return fail(FCAB_ERR_CUDA, cudaGetErrorString(e));
    return 0;
}

template <int NB>
cudaError_t launch_wgrad(const CUtensorMap &tdy, const CUtensorMap &tx, const WgArgs &a, dim3 grid,
                         cudaStream_t st)
{
    using Cfg = WgCfg<NB>;
    static bool attr_set[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (!attr_set[dev & 63]) {
        cudaError_t e = cudaFuncSetAttribute(k_conv_wgrad<NB>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, Cfg::SMEM);
        if (e != cudaSuccess)
            return e;
        attr_set[dev & 63] = true;
    }
    k_conv_wgrad<NB><<<grid, 128, Cfg::SMEM, st>>>(tdy, tx, a);
    return cudaGetLastError();
}

int grid_for(long long n)
{
    long long b = (n + 255) / 256;
    return (int)(b < 148 * 16 ? (b < 1 ? 1 : b) : 148 * 16);
}

}  // namespace unet

using namespace unet;

extern "C" {

int fcab_unet_conv_fwd(const void *x, int N, int H, int W, int Cin, const void *w, int Cout,
                       const float *bias, int relu, void *y, void *stream)
{
    return conv_gemm(x, N, H, W, Cin, w, Cout, bias, relu, y, (cudaStream_t)stream);
}

int fcab_unet_conv_dgrad(const void *dy, int N, int H, int W, int Cout, const void *wt, int Cin,
                         void *dx, void *stream)
{
    return conv_gemm(dy, N, H, W, Cout, wt, Cin, nullptr, 0, dx, (cudaStream_t)stream);
}

int fcab_unet_conv_wgrad(const void *dy, const void *x, int N, int H, int W, int Cin, int Cout,
                         float *dw, void *stream)
{
    if (N < 1 || H < 1 || W < 1 || Cin % 16 || Cout % 32)
        return fail(FCAB_ERR_ARG, "wgrad: Cin must be a multiple of 16 and Cout of 32");
    const long long P = (long long)N * (H + 2) * (W + 2);
    if (P >= (1ll << 31) - 256)
        return fail(FCAB_ERR_ARG, "wgrad: too many pixels");
    CUtensorMap tdy, tx;
    if (!make_map(&tdy, dy, P, Cout, 64, 64, CU_TENSOR_MAP_SWIZZLE_128B) ||
        !make_map(&tx, x, P, Cin, 64, 64, CU_TENSOR_MAP_SWIZZLE_128B))
        return fail(FCAB_ERR_CUDA, "wgrad: tensor map encoding failed");
    const int nb_needed = (Cin + 63) / 64;
    const int NB = nb_needed >= 4 ? 4 : nb_needed;
    const int ci_tiles = (Cin + 64 * NB - 1) / (64 * NB);
    const int co_tiles = (Cout + 127) / 128;
    const long long ksteps = (P + 63) / 64;
    // about four CTAs per SM in total
    long long want = (148LL * 4) / (9LL * co_tiles * ci_tiles);
    if (want < 1)
        want = 1;
    long long kpc = (ksteps + want - 1) / want;
    if (kpc < 8)
        kpc = 8;
    const long long splits = (ksteps + kpc - 1) / kpc;
    WgArgs a;
    a.P = (int)P;
    a.Wp = W + 2;
    a.Cin = Cin;
    a.Cout = Cout;
    a.kpc = (int)kpc;
    a.dw = dw;
    dim3 grid((unsigned)splits, (unsigned)(9 * co_tiles), (unsigned)ci_tiles);
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = NB == 1   ? launch_wgrad<1>(tdy, tx, a, grid, st)
                    : NB == 2 ? launch_wgrad<2>(tdy, tx, a, grid, st)
                    : NB == 3 ? launch_wgrad<3>(tdy, tx, a, grid, st)
                              : launch_wgrad<4>(tdy, tx, a, grid, st);
    if (e != cudaSuccess)
        return fail(FCAB_ERR_CUDA, cudaGetErrorString(e));
    return 0;
}

#define FCAB_EW_LAUNCH(kern, n, ...)                                                   \
    do {                                                                               \
        kern<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(__VA_ARGS__);              \
        cudaError_t e_ = cudaGetLastError();                                           \
        if (e_ != cudaSuccess)                                                         \
            return fail(FCAB_ERR_CUDA, cudaGetErrorString(e_));                        \
        return 0;                                                                      \
    } while (0)

int fcab_unet_maxpool2(const void *x, void *y, uint8_t *idx, int N, int H, int W, int C, void *stream)
{
    if (H % 2 || W % 2)
        return fail(FCAB_ERR_ARG, "maxpool2: H and W must be even");
    FCAB_EW_LAUNCH(k_maxpool2, (long long)N * (H / 2) * (W / 2) * C, (const bf16 *)x, (bf16 *)y, idx,
                   N, H, W, C);
}

int fcab_unet_maxpool2_bwd(const void *dy, const uint8_t *idx, void *dx, int N, int H, int W, int C,
                           void *stream)
{
    FCAB_EW_LAUNCH(k_maxpool2_bwd, (long long)N * (H / 2) * (W / 2) * C, (const bf16 *)dy, idx,
                   (bf16 *)dx, N, H, W, C);
}

int fcab_unet_upsample2(const void *x, void *y, int N, int H, int W, int C, void *stream)
{
    FCAB_EW_LAUNCH(k_upsample2, (long long)N * 4 * H * W * C, (const bf16 *)x, (bf16 *)y, N, H, W, C);
}

int fcab_unet_upsample2_bwd(const void *dy, void *dx, int N, int H, int W, int C, void *stream)
{
    FCAB_EW_LAUNCH(k_upsample2_bwd, (long long)N * H * W * C, (const bf16 *)dy, (bf16 *)dx, N, H, W, C);
}

int fcab_unet_concat(const void *a, int Ca, const void *b, int Cb, void *y, int N, int H, int W,
                     int backward, void *stream)
{
    FCAB_EW_LAUNCH(k_concat, (long long)N * H * W * (Ca + Cb), (const bf16 *)a, Ca, (const bf16 *)b,
                   Cb, (bf16 *)y, N, H, W, backward);
}

int fcab_unet_add(void *y, const void *x, long long n, void *stream)
{
    FCAB_EW_LAUNCH(k_add, n, (bf16 *)y, (const bf16 *)x, n);
}

int fcab_unet_relu_bwd(void *g, const void *y, long long n, void *stream)
{
    FCAB_EW_LAUNCH(k_relu_bwd, n, (bf16 *)g, (const bf16 *)y, n);
}

int fcab_unet_dropout(void *x, long long n, float p, uint32_t seed, void *stream)
{
    if (!(p >= 0.0f && p < 1.0f))
        return fail(FCAB_ERR_ARG, "dropout: p must be in [0, 1)");
    FCAB_EW_LAUNCH(k_dropout, n, (bf16 *)x, n, p, seed);
}

int fcab_unet_bias_grad(const void *g, long long P, int C, float *db, void *stream)
{
    if (C < 1 || C > 256)
        return fail(FCAB_ERR_ARG, "bias_grad: C must be in 1..256");
    const int lanes = 256 / C;
    long long blocks = (P + lanes * 64 - 1) / (lanes * 64);
    if (blocks > 148 * 8)
        blocks = 148 * 8;
    k_bias_grad<<<(unsigned)(blocks < 1 ? 1 : blocks), lanes * C, 0, (cudaStream_t)stream>>>(
        (const bf16 *)g, P, C, db);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : fail(FCAB_ERR_CUDA, cudaGetErrorString(e));
}

int fcab_unet_head_fwd(const void *x, const float *w, const float *b, float *out, int N, int H,
                       int W, int C, void *stream)
{
    FCAB_EW_LAUNCH(k_head_fwd, (long long)N * H * W, (const bf16 *)x, w, b, out, N, H, W, C);
}

int fcab_unet_head_bwd(const void *x, const float *w, const float *out, const float *target,
                       void *dx, float *dw, float *db, float *loss, int N, int H, int W, int C,
                       void *stream)
{
    if (C > 256)
        return fail(FCAB_ERR_ARG, "head: C must be <= 256");
    const float inv = 1.0f / (float)((long long)N * H * W);
    FCAB_EW_LAUNCH(k_head_bwd, (long long)N * H * W, (const bf16 *)x, w, out, target, (bf16 *)dx, dw,
                   db, loss, N, H, W, C, inv);
}

int fcab_unet_prep_weights(const float *w, void *wb, void *wt, int Cout, int Cin, void *stream)
{
    FCAB_EW_LAUNCH(k_prep_weights, (long long)Cout * 9 * Cin, w, (bf16 *)wb, (bf16 *)wt, Cout, Cin);
}

int fcab_unet_adam(float *w, const float *g, float *m, float *v, long long n, float lr, float b1,
                   float b2, float eps, int t, float wd, void *stream)
{
    const float c1 = 1.0f - powf(b1, (float)t), c2 = 1.0f - powf(b2, (float)t);
    FCAB_EW_LAUNCH(k_adam, n, w, g, m, v, n, lr, b1, b2, eps, c1, c2, wd);
}

int fcab_unet_pack_input(const float *in, int Cs, void *x, int C, int N, int H, int W, void *stream)
{
    if (Cs > C)
        return fail(FCAB_ERR_ARG, "pack_input: more source channels than matrix channels");
    FCAB_EW_LAUNCH(k_pack_input, (long long)N * H * W * C, in, Cs, (bf16 *)x, C, N, H, W);
}

// Returns and clears the device error code of the surrogate kernels (0: none).
int fcab_unet_device_error(void)
{
    int v = 0, z = 0;
    if (cudaMemcpyFromSymbol(&v, g_err, sizeof(int)) != cudaSuccess)
        return -1;
    if (v)
        cudaMemcpyToSymbol(g_err, &z, sizeof(int));
    return v;
}

}  // extern "C"
