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
#include <cuda_bf16.h>

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
