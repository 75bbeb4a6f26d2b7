// BF16 GEMM on the 5th-generation tensor cores (tcgen05, TMEM accumulators)
// and the elementwise kernels of the beam-trajectory surrogate MLP (forward,
// backward, Adam).
//
//   C = A B^T (+ bias), A: M x K, B: N x K (BF16, arbitrary strides),
//   FP32 accumulation in tensor memory, epilogue: FP32 pre-activation and/or
//   BF16 activation (identity or SiLU).
//
// One CTA (4 warps) per 128-row tile; K is staged through shared memory in
// chunks of KC in the canonical K-major no-swizzle layout (8 x 16-byte core
// matrices; LBO = next core along K, SBO = next 8-row group).  One elected
// thread issues tcgen05.mma (M = 128, N <= 256, K = 16 per instruction) and
// commits to an mbarrier; the others wait on it with a bounded spin.  Warp w
// reads TMEM lanes 32w..32w+31 (its rows) with tcgen05.ld.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "common.cuh"

namespace msgb {
namespace {

constexpr int GM = 128;
constexpr int KC = 64;
constexpr int GT = 128;

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Element offset of (r, k) in a canonical K-major tile with kt columns.
__device__ __forceinline__ int canon(int r, int k, int kt) {
    return (((r >> 3) * (kt >> 3) + (k >> 3)) << 6) + ((r & 7) << 3) + (k & 7);
}

__device__ __forceinline__ uint64_t make_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version for sm_100
    return d;                // base offset 0, no swizzle
}

__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }

struct GemmArgs {
    const __nv_bfloat16 *A;
    int64_t sAm, sAk;
    const __nv_bfloat16 *B;
    int64_t sBn, sBk;
    int M, N, K;
    const float *bias;
    int act;
    float *C32;
    int64_t ldc32;
    __nv_bfloat16 *C16;
    int64_t ldc16;
    int *err;
};

__global__ void __launch_bounds__(GT) gemm_tc_kernel(GemmArgs g) {
    extern __shared__ __align__(1024) uint8_t smem[];
    __nv_bfloat16 *sA = reinterpret_cast<__nv_bfloat16 *>(smem);
    __nv_bfloat16 *sB = sA + GM * KC;
    uint64_t *mbar = reinterpret_cast<uint64_t *>(sB + 256 * KC);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(mbar + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * GM;
    const int N = g.N;
    const uint32_t ncols = N <= 32 ? 32u : (N <= 64 ? 64u : (N <= 128 ? 128u : 256u));
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(ncols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(mbar)));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = *tslot;
    const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(GM >> 4) << 24);
    const uint32_t sbo = (KC / 8) * 128;
    uint32_t phase = 0;
    bool ok = true;
    const int nchunks = (g.K + KC - 1) / KC;
    for (int c = 0; c < nchunks; ++c) {
        const int k0 = c * KC;
        for (int e = tid; e < GM * KC; e += GT) {
            const int r = e / KC, k = e % KC;
            const int gm = m0 + r, gk = k0 + k;
            sA[canon(r, k, KC)] = (gm < g.M && gk < g.K) ? g.A[gm * g.sAm + gk * g.sAk] : __float2bfloat16(0.0f);
        }
        for (int e = tid; e < N * KC; e += GT) {
            const int n = e / KC, k = e % KC;
            const int gk = k0 + k;
            sB[canon(n, k, KC)] = gk < g.K ? g.B[n * g.sBn + gk * g.sBk] : __float2bfloat16(0.0f);
        }
        asm volatile("fence.proxy.async.shared::cta;");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;");
            const int nks = min(KC, g.K - k0 + 15) / 16;
            for (int ks = 0; ks < nks && ks < KC / 16; ++ks) {
                const uint64_t da = make_desc(smem_u32(sA) + 256u * ks, 128u, sbo);
                const uint64_t db = make_desc(smem_u32(sB) + 256u * ks, 128u, sbo);
                const uint32_t accum = (c > 0 || ks > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
                    "l"(da), "l"(db), "r"(idesc), "r"(accum));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                smem_u32(mbar)));
        }
        // bounded wait for this chunk's MMAs before the tile is overwritten
        uint32_t done = 0;
        for (int it = 0; it < (1 << 22) && !done; ++it) {
            asm volatile(
                "{\n\t.reg .pred p;\n\tmbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                "selp.u32 %0, 1, 0, p;\n\t}\n"
                : "=r"(done)
                : "r"(smem_u32(mbar)), "r"(phase));
            if (!done) __nanosleep(20);
        }
        if (!done) ok = false;
        phase ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;");
        __syncthreads();
        if (!ok) break;
    }
    if (!ok) {
        if (tid == 0 && g.err) atomicOr(g.err, 1);
    } else {
        const int row = m0 + 32 * warp + lane;
        for (int col0 = 0; col0 < N; col0 += 16) {
            uint32_t r[16];
            const uint32_t taddr = tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)col0;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
                "[%16];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                  "=r"(r[15])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;");
            if (row < g.M) {
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const int col = col0 + j;
                    if (col >= N) break;
                    float z = __uint_as_float(r[j]) + (g.bias ? g.bias[col] : 0.0f);
                    if (g.C32) g.C32[row * g.ldc32 + col] = z;
                    if (g.C16) g.C16[row * g.ldc16 + col] = __float2bfloat16(g.act == 1 ? silu(z) : z);
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols));
    }
}

// ---------------------------------------------------------------------------
// TMA-fed persistent GEMM for K-contiguous operands with K <= 256 (every layer
// of the surrogate's forward pass): C = A B^T (+ bias, act).
//
// Warp roles (192 threads, one CTA per SM):
//   warp 0   - one lane issues the TMA loads: B (N x K, the layer's weights)
//              once into shared memory, where it stays for every tile; A in
//              128 x 64 chunks through a 4-stage ring (full / empty mbarriers);
//   warp 1   - one lane issues tcgen05.mma (M = 128, N, K = 16 per
//              instruction) into one of two TMEM accumulators (2 x 256
//              columns) and commits each stage back to the ring;
//   warps 2-9 - the epilogue, two warps per quarter of the TMEM lanes (a
//              warp reads only its own quarter), each taking every other
//              16-column chunk: tcgen05.ld, bias, SiLU, FP32 / BF16 stores,
//              then release the accumulator, so the MMAs of the next tile
//              overlap this tile's epilogue.
// Operands use the 128-byte swizzle (TMA box rows of 64 BF16 = 128 B); the
// UMMA descriptors address 8-row atoms of 1024 B (SBO) and advance 32 B per
// K = 16 step inside the swizzled row.  Every mbarrier wait is bounded: on
// timeout the kernel raises the error flag, lets its issued copies land,
// frees TMEM and returns.
constexpr int TG_BM = 128;
constexpr int TG_BK = 64;
constexpr int TG_STAGES = 4;
constexpr int TG_MAXKB = 4;  // K <= 256
constexpr int TG_THREADS = 320;
constexpr uint32_t TG_A_STAGE = TG_BM * TG_BK * 2;  // 16 KB
constexpr size_t TG_SMEM = (size_t)TG_STAGES * TG_A_STAGE + (size_t)TG_MAXKB * 256 * TG_BK * 2 + 256 + 1024;

struct TmaGemmArgs {
    int M, N, K, kb, n_tiles;
    const float *bias;
    int act;
    float *C32;
    int64_t ldc32;
    __nv_bfloat16 *C16;
    int64_t ldc16;
    int *err;
};

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    return done != 0;
}

// Bounded wait for the phase of the given parity; false on timeout or when
// another role has aborted.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int *abort) {
    for (int it = 0; it < (1 << 22); ++it) {
        if (mbar_try(bar, parity)) return true;
        if ((it & 63) == 63) {
            if (*abort) return false;
            __nanosleep(64);
        }
    }
    return false;
}

__device__ __forceinline__ uint64_t sw128_desc(uint32_t addr) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)1 << 16;                 // LBO (unused with the 128-byte swizzle)
    d |= (uint64_t)(1024u >> 4) << 32;      // SBO: next 8-row atom
    d |= (uint64_t)1 << 46;                 // descriptor version for sm_100
    d |= (uint64_t)2 << 61;                 // 128-byte swizzle
    return d;
}

__global__ void __launch_bounds__(TG_THREADS, 1)
gemm_tma_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, TmaGemmArgs g) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint8_t *sA = smem;
    uint8_t *sB = smem + TG_STAGES * TG_A_STAGE;
    uint64_t *bars = (uint64_t *)(sB + TG_MAXKB * 256 * TG_BK * 2);
    // bars: full[4], empty[4], bfull, tfull[2], tempty[2], mma_done
    uint32_t *tslot = (uint32_t *)(bars + 14);
    volatile int *abort = (volatile int *)(tslot + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t b_full = smem_u32(bars + 8);
    auto full = [&](int s) { return smem_u32(bars + s); };
    auto empty = [&](int s) { return smem_u32(bars + 4 + s); };
    auto tfull = [&](int a) { return smem_u32(bars + 9 + a); };
    auto tempty = [&](int a) { return smem_u32(bars + 11 + a); };
    const uint32_t mma_done = smem_u32(bars + 13);
    const uint32_t bbytes = (uint32_t)g.N * TG_BK * 2;

    if (tid == 0) {
        for (int s = 0; s < TG_STAGES; ++s) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(full(s)));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(empty(s)));
        }
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(b_full));
        for (int a = 0; a < 2; ++a) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tfull(a)));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 8;" ::"r"(tempty(a)));
        }
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mma_done));
        *abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;");
        asm volatile("prefetch.tensormap [%0];" ::"l"((uint64_t)&tmA) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"((uint64_t)&tmB) : "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(smem_u32(tslot)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = *tslot;
    const int n_local = g.n_tiles > (int)blockIdx.x ? (g.n_tiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;

    if (warp == 0) {
        if (lane == 0) {
            bool ok = true;
            // weights once
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b_full),
                         "r"(bbytes * g.kb) : "memory");
            for (int c = 0; c < g.kb; ++c)
                asm volatile(
                    "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
                    "[%4];" ::"r"(smem_u32(sB + (size_t)c * bbytes)),
                    "l"((uint64_t)&tmB), "r"(c * TG_BK), "r"(0), "r"(b_full)
                    : "memory");
            int q = 0;
            for (int it = 0; it < n_local && ok; ++it) {
                const int m0 = ((int)blockIdx.x + it * (int)gridDim.x) * TG_BM;
                for (int c = 0; c < g.kb; ++c, ++q) {
                    const int s = q % TG_STAGES, round = q / TG_STAGES;
                    if (!mbar_wait(empty(s), (round & 1) ^ 1, abort)) {
                        ok = false;
                        break;
                    }
                    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(full(s)),
                                 "r"(TG_A_STAGE) : "memory");
                    asm volatile(
                        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, "
                        "%3}], [%4];" ::"r"(smem_u32(sA + (size_t)s * TG_A_STAGE)),
                        "l"((uint64_t)&tmA), "r"(c * TG_BK), "r"(m0), "r"(full(s))
                        : "memory");
                }
            }
            if (!ok) {
                *abort = 1;
                if (g.err) atomicOr(g.err, 1);
            }
            // every issued load lands before the CTA can exit
            volatile int never = 0;
            mbar_wait(b_full, 0, &never);
            for (int k = q - TG_STAGES; k < q; ++k)
                if (k >= 0) mbar_wait(full(k % TG_STAGES), (k / TG_STAGES) & 1, &never);
        }
    } else if (warp == 1) {
        if (lane == 0) {
            bool ok = mbar_wait(b_full, 0, abort);
            const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(g.N >> 3) << 17) |
                                   ((uint32_t)(TG_BM >> 4) << 24);
            int q = 0;
            for (int it = 0; it < n_local && ok; ++it) {
                const int a = it & 1, use = it >> 1;
                if (!mbar_wait(tempty(a), (use & 1) ^ 1, abort)) {
                    ok = false;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;");
                const uint32_t dtm = tmem + (uint32_t)(a * 256);
                for (int c = 0; c < g.kb; ++c, ++q) {
                    const int s = q % TG_STAGES, round = q / TG_STAGES;
                    if (!mbar_wait(full(s), round & 1, abort)) {
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;");
                    const uint32_t abase = smem_u32(sA + (size_t)s * TG_A_STAGE);
                    const uint32_t bbase = smem_u32(sB + (size_t)c * bbytes);
#pragma unroll
                    for (int kk = 0; kk < TG_BK / 16; ++kk) {
                        const uint64_t da = sw128_desc(abase + 32u * kk);
                        const uint64_t db = sw128_desc(bbase + 32u * kk);
                        const uint32_t accum = (c > 0 || kk > 0) ? 1u : 0u;
                        asm volatile(
                            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dtm),
                            "l"(da), "l"(db), "r"(idesc), "r"(accum));
                    }
                    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                        empty(s)) : "memory");
                }
                if (!ok) break;
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                    tfull(a)) : "memory");
            }
            if (!ok) {
                *abort = 1;
                if (g.err) atomicOr(g.err, 1);
            }
            // every issued MMA has finished before TMEM is released
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                mma_done) : "memory");
            volatile int never = 0;
            mbar_wait(mma_done, 0, &never);
        }
    } else {
        const int quarter = warp & 3;         // TMEM lanes 32 quarter .. + 31
        const int half = (warp - 2) >> 2;     // 16-column chunks half, half + 2, ...
        const bool vec32 = g.C32 && (g.ldc32 & 3) == 0 && ((uintptr_t)g.C32 & 15) == 0;
        const bool vec16 = g.C16 && (g.ldc16 & 7) == 0 && ((uintptr_t)g.C16 & 15) == 0;
        bool ok = true;
        for (int it = 0; it < n_local && ok; ++it) {
            const int a = it & 1, use = it >> 1;
            const int m0 = ((int)blockIdx.x + it * (int)gridDim.x) * TG_BM;
            ok = mbar_wait(tfull(a), use & 1, abort);
            __syncwarp();
            ok = __all_sync(0xffffffffu, ok);
            if (!ok) break;
            asm volatile("tcgen05.fence::after_thread_sync;");
            const int row = m0 + 32 * quarter + lane;
            for (int col0 = 16 * half; col0 < g.N; col0 += 32) {
                uint32_t r[16];
                const uint32_t taddr = tmem + ((uint32_t)(32 * quarter) << 16) + (uint32_t)(a * 256 + col0);
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
                    "[%16];"
                    : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                      "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                      "=r"(r[15])
                    : "r"(taddr));
                asm volatile("tcgen05.wait::ld.sync.aligned;");
                if (row < g.M) {
                    float z[16];
#pragma unroll
                    for (int j = 0; j < 16; ++j) z[j] = __uint_as_float(r[j]) + (g.bias ? g.bias[col0 + j] : 0.0f);
                    // a lane's 16 columns are contiguous in its row: 16-byte stores
                    // where the output's base and row stride allow them
                    if (g.C32) {
                        float *dst = g.C32 + row * g.ldc32 + col0;
                        if (vec32) {
#pragma unroll
                            for (int j = 0; j < 16; j += 4)
                                *reinterpret_cast<float4 *>(dst + j) = make_float4(z[j], z[j + 1], z[j + 2], z[j + 3]);
                        } else {
#pragma unroll
                            for (int j = 0; j < 16; ++j) dst[j] = z[j];
                        }
                    }
                    if (g.C16) {
                        uint32_t h[8];
#pragma unroll
                        for (int j = 0; j < 8; ++j) {
                            const float u = g.act == 1 ? silu(z[2 * j]) : z[2 * j];
                            const float v = g.act == 1 ? silu(z[2 * j + 1]) : z[2 * j + 1];
                            const __nv_bfloat162 b2 = __floats2bfloat162_rn(u, v);  // .x = u (lower address)
                            h[j] = *reinterpret_cast<const uint32_t *>(&b2);
                        }
                        __nv_bfloat16 *dst = g.C16 + row * g.ldc16 + col0;
                        if (vec16) {
                            reinterpret_cast<uint4 *>(dst)[0] = make_uint4(h[0], h[1], h[2], h[3]);
                            reinterpret_cast<uint4 *>(dst)[1] = make_uint4(h[4], h[5], h[6], h[7]);
                        } else {
#pragma unroll
                            for (int j = 0; j < 8; ++j) {
                                const __nv_bfloat162 b2 = *reinterpret_cast<const __nv_bfloat162 *>(&h[j]);
                                dst[2 * j] = b2.x;
                                dst[2 * j + 1] = b2.y;
                            }
                        }
                    }
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;");
            __syncwarp();
            if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(tempty(a)) : "memory");
        }
        if (!ok && lane == 0) {
            *abort = 1;
            if (g.err) atomicOr(g.err, 1);
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem));
    }
}

// Host: cuTensorMapEncodeTiled from the driver, looked up once.
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static std::once_flag once;
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    });
    return fn;
}

// Row-major BF16 matrix (rows x K, row stride ld elements) as a 2D tensor map
// with boxes of `box_rows` x 64 and the 128-byte swizzle.
bool bf16_tensor_map(CUtensorMap *map, const void *base, int64_t rows, int64_t K, int64_t ld, int box_rows) {
    auto enc = tensor_map_encoder();
    if (!enc) return false;
    cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
    cuuint32_t box[2] = {(cuuint32_t)TG_BK, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    return enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(base), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// dZ = dA * silu'(Z) (FP32 in, BF16 and FP32 out).
__global__ void silu_backward_kernel(const float *dA, const float *Z, int64_t n, float *dZ32, __nv_bfloat16 *dZ16) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float z = Z[i];
    const float s = 1.0f / (1.0f + __expf(-z));
    const float d = dA[i] * (s * (1.0f + z * (1.0f - s)));
    if (dZ32) dZ32[i] = d;
    if (dZ16) dZ16[i] = __float2bfloat16(d);
}

// Column sums of an M x N FP32 matrix, one thread per column, fixed order.
__global__ void colsum_kernel(const float *X, int M, int N, int64_t ld, float *out) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    double s = 0.0;
    for (int m = 0; m < M; ++m) s += X[m * ld + n];
    out[n] = (float)s;
}

__global__ void adam_kernel(float *w, const float *g, float *m1, float *m2, int64_t n, float lr, float b1, float b2,
                            float eps, float bc1, float bc2, __nv_bfloat16 *w16) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float a = b1 * m1[i] + (1.0f - b1) * gi;
    const float b = b2 * m2[i] + (1.0f - b2) * gi * gi;
    m1[i] = a;
    m2[i] = b;
    const float wi = w[i] - lr * (a / bc1) / (sqrtf(b / bc2) + eps);
    w[i] = wi;
    if (w16) w16[i] = __float2bfloat16(wi);
}

__global__ void to_bf16_kernel(const float *x, int64_t n, __nv_bfloat16 *y) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) y[i] = __float2bfloat16(x[i]);
}

}  // namespace
}  // namespace msgb

using namespace msgb;

extern "C" int msgb_gemm_bf16(const msgb_gemm *p, msgb_stream_t stream) {
    if (!p || !p->A || !p->B) return fail(MSGB_ERR_ARG, "msgb_gemm_bf16: NULL operand");
    if (p->M <= 0 || p->K <= 0) return fail(MSGB_ERR_ARG, "msgb_gemm_bf16: M and K must be positive");
    if (p->N < 16 || p->N > 256 || p->N % 16) return fail(MSGB_ERR_UNSUPPORTED, "msgb_gemm_bf16: N must be a multiple of 16 in [16, 256]");
    if (!p->C32 && !p->C16) return fail(MSGB_ERR_ARG, "msgb_gemm_bf16: no output");
    if (p->act != 0 && p->act != 1) return fail(MSGB_ERR_ARG, "msgb_gemm_bf16: act must be 0 or 1");
    GemmArgs g{};
    g.A = (const __nv_bfloat16 *)p->A;
    g.sAm = p->sAm;
    g.sAk = p->sAk;
    g.B = (const __nv_bfloat16 *)p->B;
    g.sBn = p->sBn;
    g.sBk = p->sBk;
    g.M = p->M;
    g.N = p->N;
    g.K = p->K;
    g.bias = p->bias;
    g.act = p->act;
    g.C32 = p->C32;
    g.ldc32 = p->ldc32;
    g.C16 = (__nv_bfloat16 *)p->C16;
    g.ldc16 = p->ldc16;
    g.err = p->error_flag;
    // K-contiguous operands with 16-byte aligned rows and K <= 256: the TMA-fed
    // persistent kernel; other layouts (the weight-gradient products) stage
    // element by element.
    const bool tma = p->sAk == 1 && p->sBk == 1 && p->K <= TG_MAXKB * TG_BK && p->sAm >= p->K && p->sBn >= p->K &&
                     (p->sAm % 8) == 0 && (p->sBn % 8) == 0 && ((uintptr_t)p->A % 16) == 0 &&
                     ((uintptr_t)p->B % 16) == 0 && p->M < (1 << 30);
    if (tma) {
        CUtensorMap ta, tb;
        if (bf16_tensor_map(&ta, p->A, p->M, p->K, p->sAm, TG_BM) &&
            bf16_tensor_map(&tb, p->B, p->N, p->K, p->sBn, p->N)) {
            TmaGemmArgs t{};
            t.M = p->M;
            t.N = p->N;
            t.K = p->K;
            t.kb = (p->K + TG_BK - 1) / TG_BK;
            t.n_tiles = (p->M + TG_BM - 1) / TG_BM;
            t.bias = p->bias;
            t.act = p->act;
            t.C32 = p->C32;
            t.ldc32 = p->ldc32;
            t.C16 = (__nv_bfloat16 *)p->C16;
            t.ldc16 = p->ldc16;
            t.err = p->error_flag;
            cudaError_t e = cudaFuncSetAttribute(gemm_tma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 (int)TG_SMEM);
            if (e != cudaSuccess) return fail(MSGB_ERR_CUDA, "msgb_gemm_bf16: %s", cudaGetErrorString(e));
            int dev = 0, sms = 148;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            const unsigned grid = (unsigned)(t.n_tiles < sms ? t.n_tiles : sms);
            gemm_tma_kernel<<<grid, TG_THREADS, TG_SMEM, as_stream(stream)>>>(ta, tb, t);
            return check_launch("msgb_gemm_bf16");
        }
    }
    const size_t smem = sizeof(__nv_bfloat16) * (GM + 256) * KC + 16;
    cudaError_t e = cudaFuncSetAttribute(gemm_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return fail(MSGB_ERR_CUDA, "msgb_gemm_bf16: %s", cudaGetErrorString(e));
    const unsigned grid = (unsigned)((p->M + GM - 1) / GM);
    gemm_tc_kernel<<<grid, GT, smem, as_stream(stream)>>>(g);
    return check_launch("msgb_gemm_bf16");
}

extern "C" int msgb_silu_backward(const float *dA, const float *Z, int64_t n, float *dZ32, void *dZ16,
                                  msgb_stream_t stream) {
    if (!dA || !Z || (!dZ32 && !dZ16)) return fail(MSGB_ERR_ARG, "msgb_silu_backward: NULL argument");
    if (n <= 0) return MSGB_OK;
    silu_backward_kernel<<<(unsigned)((n + 255) / 256), 256, 0, as_stream(stream)>>>(dA, Z, n, dZ32,
                                                                                    (__nv_bfloat16 *)dZ16);
    return check_launch("msgb_silu_backward");
}

extern "C" int msgb_colsum(const float *X, int M, int N, int64_t ld, float *out, msgb_stream_t stream) {
    if (!X || !out || M < 0 || N <= 0) return fail(MSGB_ERR_ARG, "msgb_colsum: bad argument");
    colsum_kernel<<<(unsigned)((N + 127) / 128), 128, 0, as_stream(stream)>>>(X, M, N, ld, out);
    return check_launch("msgb_colsum");
}

extern "C" int msgb_adam(float *w, const float *g, float *m1, float *m2, int64_t n, double lr, double b1, double b2,
                         double eps, int64_t step, void *w16, msgb_stream_t stream) {
    if (!w || !g || !m1 || !m2 || step < 1) return fail(MSGB_ERR_ARG, "msgb_adam: bad argument");
    if (n <= 0) return MSGB_OK;
    const float bc1 = (float)(1.0 - pow(b1, (double)step)), bc2 = (float)(1.0 - pow(b2, (double)step));
    adam_kernel<<<(unsigned)((n + 255) / 256), 256, 0, as_stream(stream)>>>(w, g, m1, m2, n, (float)lr, (float)b1,
                                                                           (float)b2, (float)eps, bc1, bc2,
                                                                           (__nv_bfloat16 *)w16);
    return check_launch("msgb_adam");
}

extern "C" int msgb_to_bf16(const float *x, int64_t n, void *y, msgb_stream_t stream) {
    if (!x || !y) return fail(MSGB_ERR_ARG, "msgb_to_bf16: NULL argument");
    if (n <= 0) return MSGB_OK;
    to_bf16_kernel<<<(unsigned)((n + 255) / 256), 256, 0, as_stream(stream)>>>(x, n, (__nv_bfloat16 *)y);
    return check_launch("msgb_to_bf16");
}
