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

// Waits for the phase with the given parity; gives up after `limit` cycles
// (2^32 by default, about 2 s).
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, long long limit = 1ll << 32)
{
    const long long t0 = clock64();
    while (!mbar_try(bar, parity)) {
        if (clock64() - t0 > limit)
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

// The conv kernels' bounded wait on a barrier whose phase never completes
// (its one expected arrival never comes): the wait must give up and report.
__global__ void k_wait_probe(long long limit)
{
    __shared__ __align__(8) uint64_t bar;
    const uint32_t b = (uint32_t)__cvta_generic_to_shared(&bar);
    if (threadIdx.x == 0)
        mbar_init(b, 1);
    __syncthreads();
    if (threadIdx.x == 0 && !mbar_wait(b, 0, limit))
        set_err(10);
    __syncthreads();
}

__device__ __forceinline__ bool interior(int p, int P, int Hp, int Wp)
{
    if (p >= P)
        return false;
    const int q = p % (Hp * Wp);
    const int yy = q / Wp, xx = q - yy * Wp;
    return yy >= 1 && yy <= Hp - 2 && xx >= 1 && xx <= Wp - 2;
}

// ---------------------------------------------------------------------------
// Implicit-GEMM 3x3 convolution, persistent and warp-specialised: each CTA
// (one per SM) walks tiles of M = 128 pixels x N = BN output channels;
// K = 9 taps x Cin in blocks of CK channels.
//   warp 0      TMA producer (A blocks into a ring of up to 32 stages; the weights
//               either per block or, when small, once into resident smem)
//   warp 1      MMA issuer (one thread), accumulating into one of two TMEM
//               buffers so the epilogue of a tile overlaps the next tile
//   warps 2-9   epilogue, two warpgroups, one per TMEM buffer (tiles of
//               even / odd local index): TMEM -> bias, ReLU -> bf16 rows
//               of interior pixels (warp w reads TMEM lanes 32*(w%4)..+31)

struct GemmArgs {
    int P, Hp, Wp;          // padded pixel count, padded height and width
    int Cin;                // channels of the A matrix
    int Cout;               // channels (row width) of the output matrix
    int mtiles, ntiles;     // pixel tiles, total tiles (pixel tiles x channel tiles)
    int nkb;                // K blocks per tile (9 * Cin / CK)
    int bres;               // 1: the weights stay resident in shared memory
    int stages;             // A (or A+B) ring stages
    int stage_bytes;        // bytes per stage (multiple of 1024)
    unsigned long long m_hw, m_w;   // ceil(2^48 / (Hp*Wp)), ceil(2^48 / Wp)
    const float *bias;      // [Cout] or null
    bf16 *y;                // [P][Cout]
    int relu;
};

// A stage holds G taps of one channel block (G = 1, 3 or 9 for 64-, 32- and
// 16-channel blocks), so one barrier round trip covers at least 64 K of MMAs.
template <int CK, int BN>
struct GemmCfg {
    static constexpr int G = CK == 64 ? 1 : CK == 32 ? 3 : 9;
    static constexpr int A_BYTES = 128 * CK * 2;          // one tap
    static constexpr int B_BYTES = BN * CK * 2;
    static constexpr int B_AL = (B_BYTES + 1023) / 1024 * 1024;
    static constexpr uint32_t TCOLS = BN <= 32 ? 32 : BN <= 64 ? 64 : BN <= 128 ? 128 : 256;
};

// Descriptor of a K-major tile at shared address saddr (LBO 16 B).
template <int CK>
__device__ __forceinline__ uint64_t kdesc(uint32_t saddr)
{
    constexpr uint64_t hi = ((uint64_t)((KSw<CK>::sbo >> 4) & 0x3FFFu)) | (1ull << 14) |
                            ((uint64_t)KSw<CK>::layout << 29);
    return (hi << 32) | (uint64_t)(((saddr & 0x3FFFFu) >> 4) | (1u << 16));
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// floor(p / d) for p < 2^31, d < 2^17, given m = ceil(2^48 / d).
__device__ __forceinline__ int div_m(int p, unsigned long long m)
{
    return (int)__umul64hi((unsigned long long)p, m << 16);
}

template <int CK, int BN>
__global__ void __launch_bounds__(320, 1)
k_conv_gemm(const __grid_constant__ CUtensorMap tx, const __grid_constant__ CUtensorMap tw, GemmArgs a)
{
    using Cfg = GemmCfg<CK, BN>;
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    uint8_t *sm = smem_raw + (base - raw);
    const int S = a.stages;
    const uint32_t bres_off = (uint32_t)(S * a.stage_bytes);
    const uint32_t bar_off = bres_off + (a.bres ? (uint32_t)(a.nkb * Cfg::B_AL) : 0u);
    const uint32_t bar0 = base + bar_off;
    auto full = [&](int s) { return bar0 + 8u * s; };
    auto empty = [&](int s) { return bar0 + 8u * (S + s); };
    const uint32_t bfull = bar0 + 16u * S;
    auto tfull = [&](int b) { return bar0 + 16u * S + 8u + 8u * b; };
    auto tempty = [&](int b) { return bar0 + 16u * S + 24u + 8u * b; };
    uint32_t *tslot = (uint32_t *)(sm + bar_off + 16u * S + 40u);
    float *sbias = (float *)(sm + bar_off + 16u * S + 64u);   // [Cout]
    auto sA = [&](int s) { return base + (uint32_t)(s * a.stage_bytes); };

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int c = threadIdx.x; c < a.Cout; c += blockDim.x)
        sbias[c] = a.bias ? a.bias[c] : 0.0f;
    if (threadIdx.x == 0) {
        for (int s = 0; s < S; s++) {
            mbar_init(full(s), 1);
            mbar_init(empty(s), 1);
        }
        mbar_init(bfull, 1);
        for (int b = 0; b < 2; b++) {
            mbar_init(tfull(b), 1);
            mbar_init(tempty(b), 128);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 0)
        tmem_alloc(smem_u32(tslot), 2 * Cfg::TCOLS);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    const int cpt = a.Cin / CK;
    const int nkb = a.nkb;

    // K order: groups of G taps x one channel block; group q covers taps
    // G*(q / cpt) .. +G-1 of channel block q % cpt
    const int ngrp = nkb / Cfg::G;
    const bool one_ntile = a.ntiles == a.mtiles;
    if (warp == 0) {
        if (lane == 0) {
            if (a.bres) {
                mbar_expect_tx(bfull, (uint32_t)(nkb * Cfg::B_BYTES));
                for (int kb = 0; kb < nkb; kb++) {
                    const int tap = kb / cpt, c0 = (kb - tap * cpt) * CK;
                    tma_load_2d(base + bres_off + (uint32_t)(kb * Cfg::B_AL), &tw, bfull,
                                tap * a.Cin + c0, 0);
                }
            }
            const uint32_t tx_bytes =
                (uint32_t)(Cfg::G * (Cfg::A_BYTES + (a.bres ? 0 : Cfg::B_BYTES)));
            int s = 0;
            uint32_t ph = 0;            // ring round parity
            bool wrapped = false;       // past the first round of the ring
            bool bad = false;
            for (int tile = blockIdx.x; tile < a.ntiles && !bad; tile += gridDim.x) {
                int p0, co0;
                if (one_ntile) {
                    p0 = tile * 128;
                    co0 = 0;
                } else {
                    const int nt = tile / a.mtiles;
                    p0 = (tile - nt * a.mtiles) * 128;
                    co0 = nt * BN;
                }
                int c0 = 0, tap0 = 0;
                for (int qg = 0; qg < ngrp; qg++) {
                    if (wrapped && !mbar_wait(empty(s), ph ^ 1u)) {
                        set_err(1);
                        bad = true;
                        break;
                    }
                    mbar_expect_tx(full(s), tx_bytes);
                    const uint32_t st = sA(s);
#pragma unroll
                    for (int g = 0; g < Cfg::G; g++) {
                        const int tap = tap0 + g;
                        const int ky = tap >= 6 ? 2 : tap >= 3 ? 1 : 0;
                        const int shift = (ky - 1) * a.Wp + (tap - 3 * ky - 1);
                        tma_load_2d(st + (uint32_t)(g * Cfg::A_BYTES), &tx, full(s), c0, p0 + shift);
                        if (!a.bres)
                            tma_load_2d(st + (uint32_t)(Cfg::G * Cfg::A_BYTES + g * Cfg::B_AL), &tw,
                                        full(s), tap * a.Cin + c0, co0);
                    }
                    c0 += CK;
                    if (c0 == a.Cin) {
                        c0 = 0;
                        tap0 += Cfg::G;
                    }
                    if (++s == S) {
                        s = 0;
                        ph ^= 1u;
                        wrapped = true;
                    }
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            constexpr uint32_t idesc = idesc_bf16(128, BN, false, false);
            bool bad = a.bres && !mbar_wait(bfull, 0);
            if (bad)
                set_err(2);
            int s = 0, tl = 0;
            uint32_t ph = 0;
            for (int tile = blockIdx.x; tile < a.ntiles && !bad; tile += gridDim.x, tl++) {
                const int buf = tl & 1;
                if (tl >= 2 && !mbar_wait(tempty(buf), (uint32_t)((tl >> 1) - 1) & 1u)) {
                    set_err(2);
                    break;
                }
                tc_fence_after();
                const uint32_t d = tmem + (uint32_t)(buf * Cfg::TCOLS);
                int cb = 0, tap0 = 0;
                for (int qg = 0; qg < ngrp; qg++) {
                    if (!mbar_wait(full(s), ph)) {
                        set_err(2);
                        bad = true;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t st = sA(s);
#pragma unroll
                    for (int g = 0; g < Cfg::G; g++) {
                        const uint32_t ab = st + (uint32_t)(g * Cfg::A_BYTES);
                        const uint32_t bb =
                            a.bres ? base + bres_off + (uint32_t)(((tap0 + g) * cpt + cb) * Cfg::B_AL)
                                   : st + (uint32_t)(Cfg::G * Cfg::A_BYTES + g * Cfg::B_AL);
#pragma unroll
                        for (int kk = 0; kk < CK / 16; kk++)
                            umma_bf16(d, kdesc<CK>(ab + 32u * kk), kdesc<CK>(bb + 32u * kk), idesc,
                                      (qg | g | kk) != 0 ? 1u : 0u);
                    }
                    umma_commit(empty(s));
                    if (++cb == cpt) {
                        cb = 0;
                        tap0 += Cfg::G;
                    }
                    if (++s == S) {
                        s = 0;
                        ph ^= 1u;
                    }
                }
                umma_commit(tfull(buf));
            }
        }
    } else {
        const int q = warp & 3;                 // TMEM lane quarter of this warp
        const int grp = (warp - 2) >> 2;        // epilogue warpgroup = TMEM buffer
        const int row = q * 32 + lane;
        const int HW = a.Hp * a.Wp;
        int k = 0;
        for (int tile = blockIdx.x + grp * gridDim.x; tile < a.ntiles;
             tile += 2 * gridDim.x, k++) {
            if (!mbar_wait(tfull(grp), (uint32_t)k & 1u)) {
                set_err(3);
                break;
            }
            __syncwarp();
            tc_fence_after();
            const int p = (tile % a.mtiles) * 128 + row;
            const int co0 = (tile / a.mtiles) * BN;
            bool store = p < a.P;
            if (store) {
                const int qq = p - HW * div_m(p, a.m_hw);
                const int yy = div_m(qq, a.m_w);
                const int xx = qq - yy * a.Wp;
                store = yy >= 1 && yy <= a.Hp - 2 && xx >= 1 && xx <= a.Wp - 2;
            }
            const uint32_t t0 = tmem + (uint32_t)(grp * Cfg::TCOLS) + ((uint32_t)(q * 32) << 16);
#pragma unroll 1
            for (int c = 0; c < BN; c += 32) {
                float v[32];
                tmem_ld32(t0 + (uint32_t)c, v);
                if (store) {
                    __align__(16) bf16 o[32];
#pragma unroll
                    for (int j = 0; j < 32; j++) {
                        float x = v[j] + sbias[co0 + c + j];
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
            mbar_arrive(tempty(grp));
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
        tmem_dealloc(tmem, 2 * Cfg::TCOLS);
}

// ---------------------------------------------------------------------------
// Small-channel convolutions (16- or 32-channel K blocks): one halo'd A tile
// per super-tile of MT x 128 pixels serves all nine taps. The tile holds the
// rows p0 - Wp - 1 .. p0 + MT*128 + Wp of the activation matrix in the
// unswizzled K-major layout: 8-channel planes of 16-byte rows, 8-row groups
// 128 B apart (SBO) and planes `plane` bytes apart (LBO), i.e. plain linear
// rows, so tap (ky, kx) of tile t is the same tile read from row
// t*128 + ky*Wp + kx. Per 128 output pixels this loads (MT*128 + 2*Wp +
// 2) / MT rows instead of 9 x 128. Weights stay resident (swizzled, as in
// k_conv_gemm). Same warp roles as k_conv_gemm; TMEM holds two buffers of MT
// accumulators, TCS columns each.

struct HaloArgs {
    int P, Hp, Wp;          // padded pixel count, padded height and width
    int Cin, Cout;
    int nsup;               // super-tiles of MT x 128 pixels
    int nkb;                // channel blocks (Cin / CK)
    int rows_alloc;         // rows per 8-channel plane (multiple of 128)
    int stages;             // ring stages (one halo tile per channel block)
    int stage_bytes;        // (CK / 8) x rows_alloc x 16
    unsigned long long m_hw, m_w;   // ceil(2^48 / (Hp*Wp)), ceil(2^48 / Wp)
    const float *bias;      // [Cout] or null
    bf16 *y;                // [P][Cout]
    int relu;
};

template <int CK, int BN, int MT>
struct HaloCfg {
    static constexpr int NPL = CK / 8;                      // planes per stage
    static constexpr int B_BYTES = BN * CK * 2;
    static constexpr int B_AL = (B_BYTES + 1023) / 1024 * 1024;
    static constexpr uint32_t TCS = BN <= 32 ? 32 : BN <= 64 ? 64 : 128;   // columns per tile
    static constexpr uint32_t TCOLS = 2 * MT * TCS;         // two buffers of MT tiles
};

template <int CK, int BN, int MT>
__global__ void __launch_bounds__(320, 1)
k_conv_halo(const __grid_constant__ CUtensorMap tx, const __grid_constant__ CUtensorMap tw,
            HaloArgs a)
{
    using Cfg = HaloCfg<CK, BN, MT>;
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    uint8_t *sm = smem_raw + (base - raw);
    const int S = a.stages;
    const uint32_t plane = (uint32_t)a.rows_alloc * 16u;
    const uint32_t bres_off = (uint32_t)(S * a.stage_bytes);
    const uint32_t bar_off = bres_off + (uint32_t)(9 * a.nkb * Cfg::B_AL);
    const uint32_t bar0 = base + bar_off;
    auto full = [&](int s) { return bar0 + 8u * s; };
    auto empty = [&](int s) { return bar0 + 8u * (S + s); };
    const uint32_t bfull = bar0 + 16u * S;
    auto tfull = [&](int b) { return bar0 + 16u * S + 8u + 8u * b; };
    auto tempty = [&](int b) { return bar0 + 16u * S + 24u + 8u * b; };
    uint32_t *tslot = (uint32_t *)(sm + bar_off + 16u * S + 40u);
    float *sbias = (float *)(sm + bar_off + 16u * S + 64u);
    auto sA = [&](int s) { return base + (uint32_t)(s * a.stage_bytes); };
    auto sB = [&](int q) { return base + bres_off + (uint32_t)(q * Cfg::B_AL); };

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int c = threadIdx.x; c < a.Cout; c += blockDim.x)
        sbias[c] = a.bias ? a.bias[c] : 0.0f;
    if (threadIdx.x == 0) {
        for (int s = 0; s < S; s++) {
            mbar_init(full(s), 1);
            mbar_init(empty(s), 1);
        }
        mbar_init(bfull, 1);
        for (int b = 0; b < 2; b++) {
            mbar_init(tfull(b), 1);
            mbar_init(tempty(b), 128);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 0)
        tmem_alloc(smem_u32(tslot), Cfg::TCOLS);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    const int nkb = a.nkb;
    const int nbox = a.rows_alloc / 128;

    if (warp == 0) {
        if (lane == 0) {
            // resident weights: chunk q = tap * nkb + kb holds w[.][tap][kb*CK ..]
            mbar_expect_tx(bfull, (uint32_t)(9 * nkb * Cfg::B_BYTES));
            for (int tap = 0; tap < 9; tap++)
                for (int kb = 0; kb < nkb; kb++)
                    tma_load_2d(sB(tap * nkb + kb), &tw, bfull, tap * a.Cin + kb * CK, 0);
            const uint32_t tx_bytes = (uint32_t)(Cfg::NPL * nbox * 128 * 16);
            int s = 0;
            uint32_t ph = 0;
            bool wrapped = false, bad = false;
            for (int sup = blockIdx.x; sup < a.nsup && !bad; sup += gridDim.x) {
                const int r0 = sup * MT * 128 - a.Wp - 1;
                for (int kb = 0; kb < nkb; kb++) {
                    if (wrapped && !mbar_wait(empty(s), ph ^ 1u)) {
                        set_err(7);
                        bad = true;
                        break;
                    }
                    mbar_expect_tx(full(s), tx_bytes);
                    for (int j = 0; j < Cfg::NPL; j++)
                        for (int b = 0; b < nbox; b++)
                            tma_load_2d(sA(s) + (uint32_t)j * plane + (uint32_t)b * 2048u, &tx,
                                        full(s), kb * CK + 8 * j, r0 + 128 * b);
                    if (++s == S) {
                        s = 0;
                        ph ^= 1u;
                        wrapped = true;
                    }
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            constexpr uint32_t idesc = idesc_bf16(128, BN, false, false);
            bool bad = !mbar_wait(bfull, 0);
            if (bad)
                set_err(8);
            int s = 0, tl = 0;
            uint32_t ph = 0;
            for (int sup = blockIdx.x; sup < a.nsup && !bad; sup += gridDim.x, tl++) {
                const int buf = tl & 1;
                if (tl >= 2 && !mbar_wait(tempty(buf), (uint32_t)((tl >> 1) - 1) & 1u)) {
                    set_err(8);
                    break;
                }
                tc_fence_after();
                for (int kb = 0; kb < nkb; kb++) {
                    if (!mbar_wait(full(s), ph)) {
                        set_err(8);
                        bad = true;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t st = sA(s);
                    for (int tap = 0; tap < 9; tap++) {
                        const int ky = tap >= 6 ? 2 : tap >= 3 ? 1 : 0;
                        const uint32_t off = (uint32_t)(ky * a.Wp + (tap - 3 * ky)) * 16u;
                        const uint32_t bb = sB(tap * nkb + kb);
#pragma unroll
                        for (int t = 0; t < MT; t++) {
                            const uint32_t d = tmem + (uint32_t)((buf * MT + t) * Cfg::TCS);
#pragma unroll
                            for (int kk = 0; kk < CK / 16; kk++) {
                                // K = 16: planes 2kk (k 0-7) and 2kk+1 (k 8-15, LBO apart)
                                const uint32_t aa = st + (uint32_t)(2 * kk) * plane +
                                                    (uint32_t)(t * 128) * 16u + off;
                                umma_bf16(d, smem_desc(aa, plane, 128u, 0u),
                                          kdesc<CK>(bb + 32u * kk), idesc,
                                          (kb | tap | kk) != 0 ? 1u : 0u);
                            }
                        }
                    }
                    umma_commit(empty(s));
                    if (++s == S) {
                        s = 0;
                        ph ^= 1u;
                    }
                }
                umma_commit(tfull(buf));
            }
        }
    } else {
        const int q = warp & 3;                 // TMEM lane quarter of this warp
        const int grp = (warp - 2) >> 2;        // epilogue warpgroup = TMEM buffer
        const int row = q * 32 + lane;
        const int HW = a.Hp * a.Wp;
        int k = 0;
        for (int sup = blockIdx.x + grp * gridDim.x; sup < a.nsup; sup += 2 * gridDim.x, k++) {
            if (!mbar_wait(tfull(grp), (uint32_t)k & 1u)) {
                set_err(9);
                break;
            }
            __syncwarp();
            tc_fence_after();
#pragma unroll 1
            for (int t = 0; t < MT; t++) {
                const int p = (sup * MT + t) * 128 + row;
                bool store = p < a.P;
                if (store) {
                    const int qq = p - HW * div_m(p, a.m_hw);
                    const int yy = div_m(qq, a.m_w);
                    const int xx = qq - yy * a.Wp;
                    store = yy >= 1 && yy <= a.Hp - 2 && xx >= 1 && xx <= a.Wp - 2;
                }
                const uint32_t t0 = tmem + (uint32_t)((grp * MT + t) * Cfg::TCS) +
                                    ((uint32_t)(q * 32) << 16);
#pragma unroll 1
                for (int c = 0; c < BN; c += 32) {
                    float v[32];
                    tmem_ld32(t0 + (uint32_t)c, v);
                    if (store) {
                        __align__(16) bf16 o[32];
#pragma unroll
                        for (int j = 0; j < 32; j++) {
                            float x = v[j] + sbias[c + j];
                            if (a.relu)
                                x = fmaxf(x, 0.0f);
                            o[j] = __float2bfloat16_rn(x);
                        }
                        uint4 *dst = (uint4 *)(a.y + (size_t)p * a.Cout + c);
                        const uint4 *src = (const uint4 *)o;
#pragma unroll
                        for (int j = 0; j < 4; j++)
                            dst[j] = src[j];
                    }
                }
            }
            tc_fence_before();
            mbar_arrive(tempty(grp));
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

// Pixel-wise layers move 16-byte vectors of 8 bf16 channels (C is a
// multiple of 16); index arithmetic is per vector, in 32 bits.
__device__ __forceinline__ void unpack8(uint4 u, float (&f)[8])
{
    const __nv_bfloat162 *h = (const __nv_bfloat162 *)&u;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const float2 t = __bfloat1622float2(h[k]);
        f[2 * k] = t.x;
        f[2 * k + 1] = t.y;
    }
}

__device__ __forceinline__ uint4 pack8(const float (&f)[8])
{
    uint4 u;
    __nv_bfloat162 *h = (__nv_bfloat162 *)&u;
#pragma unroll
    for (int k = 0; k < 4; k++)
        h[k] = __floats2bfloat162_rn(f[2 * k], f[2 * k + 1]);
    return u;
}

#define FCAB_GRID_LOOP(i, total)                                                      \
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < (total); i += gridDim.x * blockDim.x)

// 2x2 max pooling of an (H, W) image (V vectors per pixel); idx keeps the
// arg max (0..3, first maximum) of every channel for the backward pass.
__global__ void k_maxpool2(const uint4 *x, uint4 *y, uint2 *idx, int N, int H, int W, int V)
{
    const int Ho = H / 2, Wo = W / 2;
    FCAB_GRID_LOOP(i, N * Ho * Wo * V)
    {
        const int v = i % V;
        int t = i / V;
        const int ox = t % Wo;
        t /= Wo;
        const int oy = t % Ho;
        const int n = t / Ho;
        float best[8], cur[8];
        uint32_t arg[8];
        unpack8(x[prow(n, 2 * oy, 2 * ox, H, W) * V + v], best);
#pragma unroll
        for (int c = 0; c < 8; c++)
            arg[c] = 0;
#pragma unroll
        for (int k = 1; k < 4; k++) {
            unpack8(x[prow(n, 2 * oy + (k >> 1), 2 * ox + (k & 1), H, W) * V + v], cur);
#pragma unroll
            for (int c = 0; c < 8; c++)
                if (cur[c] > best[c]) {
                    best[c] = cur[c];
                    arg[c] = k;
                }
        }
        y[prow(n, oy, ox, Ho, Wo) * V + v] = pack8(best);
        uint2 a;
        a.x = arg[0] | arg[1] << 8 | arg[2] << 16 | arg[3] << 24;
        a.y = arg[4] | arg[5] << 8 | arg[6] << 16 | arg[7] << 24;
        idx[i] = a;
    }
}

// Gradient of the pooling: each input pixel gets dy where it was the arg
// max, else 0; plus, when add is given, add[p][aoff + ...] (row width aV
// vectors): the skip connection's gradient taken straight from the
// concatenation's gradient.
__global__ void k_maxpool2_bwd(const uint4 *dy, const uint2 *idx, const uint4 *add, int aV, int aoff,
                               uint4 *dx, int N, int H, int W, int V)
{
    const int Ho = H / 2, Wo = W / 2;
    FCAB_GRID_LOOP(i, N * Ho * Wo * V)
    {
        const int v = i % V;
        int t = i / V;
        const int ox = t % Wo;
        t /= Wo;
        const int oy = t % Ho;
        const int n = t / Ho;
        float g[8];
        unpack8(dy[prow(n, oy, ox, Ho, Wo) * V + v], g);
        const uint2 a = idx[i];
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const long long p = prow(n, 2 * oy + (k >> 1), 2 * ox + (k & 1), H, W);
            float o[8], ad[8];
            if (add)
                unpack8(add[p * aV + aoff + v], ad);
#pragma unroll
            for (int c = 0; c < 8; c++) {
                const uint32_t ac = ((c < 4 ? a.x : a.y) >> (8 * (c & 3))) & 0xffu;
                o[c] = ac == (uint32_t)k ? g[c] : 0.0f;
                if (add)
                    o[c] += ad[c];
            }
            dx[p * V + v] = pack8(o);
        }
    }
}

// y = [a | b] over the interior pixels of an (H, W) image; a is read at
// half resolution (nearest 2x upsampling) when a_half != 0. Vb = 0 gives
// the plain upsampling.
__global__ void k_cat2(const uint4 *a, int Va, int a_half, const uint4 *b, int Vb, uint4 *y, int N,
                       int H, int W)
{
    const int V = Va + Vb;
    FCAB_GRID_LOOP(i, N * H * W * V)
    {
        const int v = i % V;
        int t = i / V;
        const int x = t % W;
        t /= W;
        const int yy = t % H;
        const int n = t / H;
        const long long r = prow(n, yy, x, H, W);
        uint4 val;
        if (v < Va)
            val = a_half ? a[prow(n, yy >> 1, x >> 1, H >> 1, W >> 1) * Va + v] : a[r * Va + v];
        else
            val = b[r * Vb + (v - Va)];
        y[r * V + v] = val;
    }
}

// Split of a concatenation's gradient y = [a | b] (same resolution).
__global__ void k_split(const uint4 *y, uint4 *a, int Va, uint4 *b, int Vb, int N, int H, int W)
{
    const int V = Va + Vb;
    FCAB_GRID_LOOP(i, N * H * W * V)
    {
        const int v = i % V;
        int t = i / V;
        const int x = t % W;
        t /= W;
        const int yy = t % H;
        const int n = t / H;
        const long long r = prow(n, yy, x, H, W);
        if (v < Va)
            a[r * Va + v] = y[r * V + v];
        else
            b[r * Vb + (v - Va)] = y[r * V + v];
    }
}

// Gradient of the nearest 2x upsampling: dx (H, W, V vectors) sums the four
// children in dy (2H, 2W; row width sV vectors, first V of them used).
__global__ void k_upsum(const uint4 *dy, int sV, uint4 *dx, int N, int H, int W, int V)
{
    FCAB_GRID_LOOP(i, N * H * W * V)
    {
        const int v = i % V;
        int t = i / V;
        const int x = t % W;
        t /= W;
        const int yy = t % H;
        const int n = t / H;
        float s[8], c[8];
#pragma unroll
        for (int j = 0; j < 8; j++)
            s[j] = 0.0f;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            unpack8(dy[prow(n, 2 * yy + (k >> 1), 2 * x + (k & 1), 2 * H, 2 * W) * sV + v], c);
#pragma unroll
            for (int j = 0; j < 8; j++)
                s[j] += c[j];
        }
        dx[prow(n, yy, x, H, W) * V + v] = pack8(s);
    }
}

// y += x (FP32 sum), n8 vectors.
__global__ void k_add(uint4 *y, const uint4 *x, long long n8)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n8;
         i += (long long)gridDim.x * blockDim.x) {
        float a[8], b[8];
        unpack8(y[i], a);
        unpack8(x[i], b);
#pragma unroll
        for (int j = 0; j < 8; j++)
            a[j] += b[j];
        y[i] = pack8(a);
    }
}

// g *= (y > 0) over the whole matrix (borders are zero in g), n8 vectors.
__global__ void k_relu_bwd(uint4 *g, const uint4 *y, long long n8)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n8;
         i += (long long)gridDim.x * blockDim.x) {
        float a[8], b[8];
        unpack8(g[i], a);
        unpack8(y[i], b);
#pragma unroll
        for (int j = 0; j < 8; j++)
            a[j] = b[j] > 0.0f ? a[j] : 0.0f;
        g[i] = pack8(a);
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

// Inverted dropout in place: element e is kept when hash(seed, e) >= p*2^32,
// kept values scaled by 1/(1-p). The backward pass regenerates the mask with
// the same seed. Border pixels stay zero.
__global__ void k_dropout(uint4 *x, long long n8, float p, uint32_t seed)
{
    const uint32_t thr = (uint32_t)(p * 4294967296.0);
    const float scale = 1.0f / (1.0f - p);
    const uint32_t hs = hash32(seed);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n8;
         i += (long long)gridDim.x * blockDim.x) {
        float a[8];
        unpack8(x[i], a);
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const long long e = i * 8 + j;
            const uint32_t h = hash32((uint32_t)e ^ hash32(hs + (uint32_t)(e >> 32) * 0x9e3779b9U));
            a[j] = h >= thr ? a[j] * scale : 0.0f;
        }
        x[i] = pack8(a);
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
template <int C>
__global__ void k_head_fwd(const uint4 *x, const float *w, const float *b, float *out, int N, int H,
                           int W)
{
    constexpr int V = C / 8;
    FCAB_GRID_LOOP(i, N * H * W)
    {
        const int xx = i % W;
        const int t = i / W;
        const int yy = t % H;
        const int n = t / H;
        const long long r = prow(n, yy, xx, H, W) * V;
        float s = b[0];
#pragma unroll
        for (int v = 0; v < V; v++) {
            float f[8];
            unpack8(x[r + v], f);
#pragma unroll
            for (int j = 0; j < 8; j++)
                s += w[v * 8 + j] * f[j];
        }
        out[i] = s;
    }
}

// Mean squared error of the head against the target, and its gradients:
// dx (bf16, bordered), dw[c], db, loss sum (accumulated). Each thread keeps
// its dw partial sums in registers; warps reduce them before the atomics.
template <int C>
__global__ void k_head_bwd(const uint4 *x, const float *w, const float *out, const float *target,
                           uint4 *dx, float *dw, float *db, float *loss, int N, int H, int W,
                           float inv_count)
{
    constexpr int V = C / 8;
    float acc[C];
#pragma unroll
    for (int c = 0; c < C; c++)
        acc[c] = 0.0f;
    float ldb = 0.0f, lloss = 0.0f;
    FCAB_GRID_LOOP(i, N * H * W)
    {
        const int xx = i % W;
        const int t = i / W;
        const int yy = t % H;
        const int n = t / H;
        const long long r = prow(n, yy, xx, H, W) * V;
        const float e = out[i] - target[i];
        lloss += e * e;
        const float d = 2.0f * e * inv_count;
        ldb += d;
#pragma unroll
        for (int v = 0; v < V; v++) {
            float f[8], o[8];
            unpack8(x[r + v], f);
#pragma unroll
            for (int j = 0; j < 8; j++) {
                acc[v * 8 + j] += d * f[j];
                o[j] = d * w[v * 8 + j];
            }
            dx[r + v] = pack8(o);
        }
    }
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int c = 0; c < C; c++) {
        float s = acc[c];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
            s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0)
            atomicAdd(dw + c, s);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        ldb += __shfl_xor_sync(0xffffffffu, ldb, o);
        lloss += __shfl_xor_sync(0xffffffffu, lloss, o);
    }
    if (lane == 0) {
        atomicAdd(db, ldb);
        atomicAdd(loss, lloss);
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

// FP32 inputs [N][H][W][Cs] -> bf16 bordered matrix with C >= Cs channels.
__global__ void k_pack_input(const float *in, int Cs, uint4 *x, int C, int N, int H, int W)
{
    const int V = C / 8;
    FCAB_GRID_LOOP(i, N * H * W * V)
    {
        const int v = i % V;
        const int t = i / V;
        const int xx = t % W;
        const int t2 = t / W;
        const int yy = t2 % H;
        const int n = t2 / H;
        float f[8];
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const int c = v * 8 + j;
            f[j] = c < Cs ? in[(long long)t * Cs + c] : 0.0f;
        }
        x[prow(n, yy, xx, H, W) * V + v] = pack8(f);
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

constexpr int SMEM_MAX = 232448;   // per-CTA dynamic shared memory limit (227 KB)

template <int CK, int BN>
cudaError_t launch_gemm(const CUtensorMap &tx, const CUtensorMap &tw, GemmArgs a, cudaStream_t st)
{
    using Cfg = GemmCfg<CK, BN>;
    // resident weights when they take at most 96 KB and there is one
    // channel tile; the A ring gets what is left (at most 8 stages)
    const int bres_bytes = a.nkb * Cfg::B_AL;
    a.bres = (a.ntiles == a.mtiles && bres_bytes <= 98304) ? 1 : 0;
    a.stage_bytes = Cfg::G * (Cfg::A_BYTES + (a.bres ? 0 : Cfg::B_AL));
    // as many stages as fit (the loads in flight hide the L2 latency of the
    // nine shifted tap tiles); barrier area 16 B per stage + 64 B
    const int fixed = 1024 + (a.bres ? bres_bytes : 0) + 64 + 4 * a.Cout;
    int stages = (SMEM_MAX - fixed) / (a.stage_bytes + 16);
    stages = stages > 32 ? 32 : stages;
    if (stages < 2)
        return cudaErrorInvalidValue;
    a.stages = stages;
    const int smem = fixed + stages * (a.stage_bytes + 16);
    static int attr_smem[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (attr_smem[dev & 63] < smem) {
        cudaError_t e = cudaFuncSetAttribute(k_conv_gemm<CK, BN>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_MAX);
        if (e != cudaSuccess)
            return e;
        attr_smem[dev & 63] = SMEM_MAX;
    }
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const int grid = a.ntiles < nsm ? a.ntiles : nsm;
    k_conv_gemm<CK, BN><<<grid, 320, smem, st>>>(tx, tw, a);
    return cudaGetLastError();
}

template <int CK>
cudaError_t gemm_bn(const CUtensorMap &tx, const CUtensorMap &tw, const GemmArgs &a, int bn,
                    cudaStream_t st)
{
    switch (bn) {
    case 32: return launch_gemm<CK, 32>(tx, tw, a, st);
    case 64: return launch_gemm<CK, 64>(tx, tw, a, st);
    case 96: return launch_gemm<CK, 96>(tx, tw, a, st);
    case 128: return launch_gemm<CK, 128>(tx, tw, a, st);
    case 192: return launch_gemm<CK, 192>(tx, tw, a, st);
    case 256: return launch_gemm<CK, 256>(tx, tw, a, st);
    default: return cudaErrorInvalidValue;
    }
}

template <int CK, int BN, int MT>
cudaError_t launch_halo(const CUtensorMap &txh, const CUtensorMap &tw, const HaloArgs &a, int smem,
                        cudaStream_t st)
{
    static bool attr_set[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (!attr_set[dev & 63]) {
        cudaError_t e = cudaFuncSetAttribute(k_conv_halo<CK, BN, MT>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_MAX);
        if (e != cudaSuccess)
            return e;
        attr_set[dev & 63] = true;
    }
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const int grid = a.nsup < nsm ? a.nsup : nsm;
    k_conv_halo<CK, BN, MT><<<grid, 320, smem, st>>>(txh, tw, a);
    return cudaGetLastError();
}

// The halo path for 16/32-channel K blocks and one output tile of at most
// 128 channels, when its tiles fit in shared memory. Returns
// cudaErrorNotSupported when the shape does not qualify (the caller then
// uses k_conv_gemm).
template <int CK>
cudaError_t try_halo(const void *x, const CUtensorMap &tw, int N, int H, int W, int Cin, int Cout,
                     const float *bias, int relu, void *y, cudaStream_t st)
{
    if (Cout > 128)
        return cudaErrorNotSupported;
    const int MT = Cout <= 64 ? 4 : 2;
    const long long P = (long long)N * (H + 2) * (W + 2);
    const int Wp = W + 2;
    const int rows = MT * 128 + 2 * Wp + 2;
    const int rows_alloc = (rows + 127) / 128 * 128;
    if (rows_alloc * 16 >= (1 << 18))          // LBO field limit
        return cudaErrorNotSupported;
    const int nkb = Cin / CK;
    const int bn_al = (Cout * CK * 2 + 1023) / 1024 * 1024;
    const int bres = 9 * nkb * bn_al;
    const int stage = (CK / 8) * rows_alloc * 16;
    const int fixed = 1024 + bres + 64 + 4 * Cout;
    int stages = (SMEM_MAX - fixed) / (stage + 16);
    stages = stages > 4 ? 4 : stages;
    if (stages < 2)
        return cudaErrorNotSupported;
    CUtensorMap txh;
    if (!make_map(&txh, x, P, Cin, 8, 128, CU_TENSOR_MAP_SWIZZLE_NONE))
        return cudaErrorInvalidValue;
    HaloArgs a;
    a.P = (int)P;
    a.Hp = H + 2;
    a.Wp = Wp;
    a.Cin = Cin;
    a.Cout = Cout;
    a.nsup = (int)((P + MT * 128 - 1) / (MT * 128));
    a.nkb = nkb;
    a.rows_alloc = rows_alloc;
    a.stages = stages;
    a.stage_bytes = stage;
    a.m_hw = ((1ull << 48) + (unsigned long long)(a.Hp * a.Wp) - 1) / (unsigned long long)(a.Hp * a.Wp);
    a.m_w = ((1ull << 48) + (unsigned long long)a.Wp - 1) / (unsigned long long)a.Wp;
    a.bias = bias;
    a.y = (bf16 *)y;
    a.relu = relu;
    const int smem = fixed + stages * (stage + 16);
    switch (Cout) {
    case 32: return launch_halo<CK, 32, 4>(txh, tw, a, smem, st);
    case 64: return launch_halo<CK, 64, 4>(txh, tw, a, smem, st);
    case 96: return launch_halo<CK, 96, 2>(txh, tw, a, smem, st);
    case 128: return launch_halo<CK, 128, 2>(txh, tw, a, smem, st);
    default: return cudaErrorNotSupported;
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
    if (P >= (1ll << 31) - 256 || (long long)(H + 2) * (W + 2) >= (1 << 17) || Cout > 384)
        return fail(FCAB_ERR_ARG, "conv: too many pixels or channels");
    const CUtensorMapSwizzle sw = CK == 64 ? CU_TENSOR_MAP_SWIZZLE_128B
                                  : CK == 32 ? CU_TENSOR_MAP_SWIZZLE_64B
                                             : CU_TENSOR_MAP_SWIZZLE_32B;
    CUtensorMap tx, tw;
    if (!make_map(&tx, x, P, Cin, CK, 128, sw) || !make_map(&tw, w, Cout, 9 * Cin, CK, bn, sw))
        return fail(FCAB_ERR_CUDA, "conv: tensor map encoding failed");
    if (CK <= 32 && bn == Cout) {
        const cudaError_t he = CK == 32 ? try_halo<32>(x, tw, N, H, W, Cin, Cout, bias, relu, y, st)
                                        : try_halo<16>(x, tw, N, H, W, Cin, Cout, bias, relu, y, st);
        if (he == cudaSuccess)
            return 0;
        if (he != cudaErrorNotSupported)
            return fail(FCAB_ERR_CUDA, cudaGetErrorString(he));
    }
    GemmArgs a;
    a.P = (int)P;
    a.Hp = H + 2;
    a.Wp = W + 2;
    a.Cin = Cin;
    a.Cout = Cout;
    a.mtiles = (int)((P + 127) / 128);
    a.ntiles = a.mtiles * (Cout / bn);
    a.nkb = 9 * (Cin / CK);
    a.bres = 0;
    a.stages = 0;
    a.stage_bytes = 0;
    a.m_hw = ((1ull << 48) + (unsigned long long)(a.Hp * a.Wp) - 1) / (unsigned long long)(a.Hp * a.Wp);
    a.m_w = ((1ull << 48) + (unsigned long long)a.Wp - 1) / (unsigned long long)a.Wp;
    a.bias = bias;
    a.y = (bf16 *)y;
    a.relu = relu;
    cudaError_t e = CK == 64 ? gemm_bn<64>(tx, tw, a, bn, st)
                    : CK == 32 ? gemm_bn<32>(tx, tw, a, bn, st)
                               : gemm_bn<16>(tx, tw, a, bn, st);
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

static bool fits32(long long n) { return n >= 0 && n < (1ll << 31); }

#define FCAB_CHECK_VEC(C, n)                                                          \
    do {                                                                              \
        if ((C) % 8 || !fits32(n))                                                    \
            return fail(FCAB_ERR_ARG, "channels must be a multiple of 8 and sizes < 2^31"); \
    } while (0)

int fcab_unet_maxpool2(const void *x, void *y, uint8_t *idx, int N, int H, int W, int C, void *stream)
{
    if (H % 2 || W % 2)
        return fail(FCAB_ERR_ARG, "maxpool2: H and W must be even");
    const long long n = (long long)N * (H / 2) * (W / 2) * (C / 8);
    FCAB_CHECK_VEC(C, n);
    FCAB_EW_LAUNCH(k_maxpool2, n, (const uint4 *)x, (uint4 *)y, (uint2 *)idx, N, H, W, C / 8);
}

int fcab_unet_maxpool2_bwd(const void *dy, const uint8_t *idx, void *dx, int N, int H, int W, int C,
                           void *stream)
{
    const long long n = (long long)N * (H / 2) * (W / 2) * (C / 8);
    FCAB_CHECK_VEC(C, n);
    FCAB_EW_LAUNCH(k_maxpool2_bwd, n, (const uint4 *)dy, (const uint2 *)idx, (const uint4 *)nullptr,
                   0, 0, (uint4 *)dx, N, H, W, C / 8);
}

int fcab_unet_maxpool2_bwd_add(const void *dy, const uint8_t *idx, const void *add, int Cadd,
                               int add_off, void *dx, int N, int H, int W, int C, void *stream)
{
    const long long n = (long long)N * (H / 2) * (W / 2) * (C / 8);
    FCAB_CHECK_VEC(C, n);
    if (Cadd % 8 || add_off % 8 || add_off + C > Cadd)
        return fail(FCAB_ERR_ARG, "maxpool2_bwd_add: bad channel slice");
    FCAB_EW_LAUNCH(k_maxpool2_bwd, n, (const uint4 *)dy, (const uint2 *)idx, (const uint4 *)add,
                   Cadd / 8, add_off / 8, (uint4 *)dx, N, H, W, C / 8);
}

int fcab_unet_upsample2(const void *x, void *y, int N, int H, int W, int C, void *stream)
{
    const long long n = (long long)N * 4 * H * W * (C / 8);
    FCAB_CHECK_VEC(C, n);
    FCAB_EW_LAUNCH(k_cat2, n, (const uint4 *)x, C / 8, 1, (const uint4 *)nullptr, 0, (uint4 *)y, N,
                   2 * H, 2 * W);
}

int fcab_unet_upsample2_bwd(const void *dy, void *dx, int N, int H, int W, int C, void *stream)
{
    const long long n = (long long)N * H * W * (C / 8);
    FCAB_CHECK_VEC(C, n);
    FCAB_EW_LAUNCH(k_upsum, n, (const uint4 *)dy, C / 8, (uint4 *)dx, N, H, W, C / 8);
}

int fcab_unet_concat(const void *a, int Ca, const void *b, int Cb, void *y, int N, int H, int W,
                     int backward, void *stream)
{
    const long long n = (long long)N * H * W * ((Ca + Cb) / 8);
    FCAB_CHECK_VEC(Ca, n);
    FCAB_CHECK_VEC(Cb, n);
    if (!backward)
        FCAB_EW_LAUNCH(k_cat2, n, (const uint4 *)a, Ca / 8, 0, (const uint4 *)b, Cb / 8, (uint4 *)y,
                       N, H, W);
    FCAB_EW_LAUNCH(k_split, n, (const uint4 *)y, (uint4 *)a, Ca / 8, (uint4 *)b, Cb / 8, N, H, W);
}

int fcab_unet_upcat(const void *coarse, int C1, const void *skip, int C2, void *y, int N, int H,
                    int W, void *stream)
{
    if (H % 2 || W % 2)
        return fail(FCAB_ERR_ARG, "upcat: H and W must be even");
    const long long n = (long long)N * H * W * ((C1 + C2) / 8);
    FCAB_CHECK_VEC(C1, n);
    FCAB_CHECK_VEC(C2, n);
    FCAB_EW_LAUNCH(k_cat2, n, (const uint4 *)coarse, C1 / 8, 1, (const uint4 *)skip, C2 / 8,
                   (uint4 *)y, N, H, W);
}

int fcab_unet_upcat_bwd(const void *gy, int C1, int C2, void *gcoarse, int N, int H, int W,
                        void *stream)
{
    if (H % 2 || W % 2)
        return fail(FCAB_ERR_ARG, "upcat_bwd: H and W must be even");
    const long long n = (long long)N * (H / 2) * (W / 2) * (C1 / 8);
    FCAB_CHECK_VEC(C1, n);
    FCAB_CHECK_VEC(C2, n);
    FCAB_EW_LAUNCH(k_upsum, n, (const uint4 *)gy, (C1 + C2) / 8, (uint4 *)gcoarse, N, H / 2, W / 2,
                   C1 / 8);
}

int fcab_unet_add(void *y, const void *x, long long n, void *stream)
{
    if (n % 8)
        return fail(FCAB_ERR_ARG, "add: n must be a multiple of 8");
    FCAB_EW_LAUNCH(k_add, n / 8, (uint4 *)y, (const uint4 *)x, n / 8);
}

int fcab_unet_relu_bwd(void *g, const void *y, long long n, void *stream)
{
    if (n % 8)
        return fail(FCAB_ERR_ARG, "relu_bwd: n must be a multiple of 8");
    FCAB_EW_LAUNCH(k_relu_bwd, n / 8, (uint4 *)g, (const uint4 *)y, n / 8);
}

int fcab_unet_dropout(void *x, long long n, float p, uint32_t seed, void *stream)
{
    if (!(p >= 0.0f && p < 1.0f) || n % 8)
        return fail(FCAB_ERR_ARG, "dropout: p must be in [0, 1) and n a multiple of 8");
    FCAB_EW_LAUNCH(k_dropout, n / 8, (uint4 *)x, n / 8, p, seed);
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
    const long long n = (long long)N * H * W;
    if (!fits32(n))
        return fail(FCAB_ERR_ARG, "head: too many pixels");
    if (C == 32)
        FCAB_EW_LAUNCH(k_head_fwd<32>, n, (const uint4 *)x, w, b, out, N, H, W);
    if (C == 64)
        FCAB_EW_LAUNCH(k_head_fwd<64>, n, (const uint4 *)x, w, b, out, N, H, W);
    return fail(FCAB_ERR_ARG, "head: C must be 32 or 64");
}

int fcab_unet_head_bwd(const void *x, const float *w, const float *out, const float *target,
                       void *dx, float *dw, float *db, float *loss, int N, int H, int W, int C,
                       void *stream)
{
    const long long n = (long long)N * H * W;
    if (!fits32(n))
        return fail(FCAB_ERR_ARG, "head: too many pixels");
    const float inv = 1.0f / (float)n;
    if (C == 32)
        FCAB_EW_LAUNCH(k_head_bwd<32>, n, (const uint4 *)x, w, out, target, (uint4 *)dx, dw, db,
                       loss, N, H, W, inv);
    if (C == 64)
        FCAB_EW_LAUNCH(k_head_bwd<64>, n, (const uint4 *)x, w, out, target, (uint4 *)dx, dw, db,
                       loss, N, H, W, inv);
    return fail(FCAB_ERR_ARG, "head: C must be 32 or 64");
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
    const long long n = (long long)N * H * W * (C / 8);
    FCAB_CHECK_VEC(C, n);
    FCAB_EW_LAUNCH(k_pack_input, n, in, Cs, (uint4 *)x, C, N, H, W);
}

// Runs the conv kernels' bounded mbarrier wait on a barrier that nothing
// arrives at, with a limit of `limit_cycles` (1 to 2^32): the wait gives up,
// the kernel records error 10 and returns.
int fcab_unet_wait_probe(long long limit_cycles, void *stream)
{
    if (limit_cycles < 1 || limit_cycles > (1ll << 32))
        return fail(FCAB_ERR_ARG, "wait_probe: limit out of range");
    k_wait_probe<<<1, 32, 0, (cudaStream_t)stream>>>(limit_cycles);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return fail(FCAB_ERR_CUDA, cudaGetErrorString(e));
    return FCAB_OK;
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
