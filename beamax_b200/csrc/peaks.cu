// Throughput probes: the denominators of the FP32, FP64 and MUFU rooflines.
//
// Each kernel runs NCH independent dependency chains per thread of one
// instruction kind, so that the pipe, not the latency, is the limit when the
// grid fills every SM.  The caller times a launch with CUDA events and divides
// msgb_peak_probe_ops() by the time.  Counting: an FMA is 2 flops (FFMA2: 4,
// two lanes of FMA); a MUFU operation is 1.
#include "common.cuh"

namespace msgb {
namespace {

constexpr int NCH = 8;  // independent chains per thread

__global__ void peak_ffma_kernel(int64_t iters, float a, float b, float *sink) {
    float x[NCH];
#pragma unroll
    for (int c = 0; c < NCH; ++c) x[c] = (float)(threadIdx.x + c) * 1e-3f;
    for (int64_t i = 0; i < iters; ++i) {
#pragma unroll
        for (int c = 0; c < NCH; ++c) x[c] = fmaf(x[c], a, b);
    }
    float s = 0.0f;
#pragma unroll
    for (int c = 0; c < NCH; ++c) s += x[c];
    sink[blockIdx.x * (int64_t)blockDim.x + threadIdx.x] = s;
}

__global__ void peak_ffma2_kernel(int64_t iters, float a, float b, float *sink) {
    float2 x[NCH];
    const float2 a2 = make_float2(a, a), b2 = make_float2(b, b);
#pragma unroll
    for (int c = 0; c < NCH; ++c) x[c] = make_float2((float)(threadIdx.x + c) * 1e-3f, (float)c * 1e-3f);
    for (int64_t i = 0; i < iters; ++i) {
#pragma unroll
        for (int c = 0; c < NCH; ++c) x[c] = __ffma2_rn(x[c], a2, b2);
    }
    float s = 0.0f;
#pragma unroll
    for (int c = 0; c < NCH; ++c) s += x[c].x + x[c].y;
    sink[blockIdx.x * (int64_t)blockDim.x + threadIdx.x] = s;
}

__global__ void peak_dfma_kernel(int64_t iters, double a, double b, float *sink) {
    double x[NCH];
#pragma unroll
    for (int c = 0; c < NCH; ++c) x[c] = (double)(threadIdx.x + c) * 1e-3;
    for (int64_t i = 0; i < iters; ++i) {
#pragma unroll
        for (int c = 0; c < NCH; ++c) x[c] = fma(x[c], a, b);
    }
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < NCH; ++c) s += x[c];
    sink[blockIdx.x * (int64_t)blockDim.x + threadIdx.x] = (float)s;
}

// x <- sin(x): MUFU.SIN chains (the summation's sincos and exp use the same unit).
__global__ void peak_mufu_kernel(int64_t iters, float *sink) {
    float x[NCH];
#pragma unroll
    for (int c = 0; c < NCH; ++c) x[c] = (float)(threadIdx.x + c) * 1e-3f + 0.5f;
    for (int64_t i = 0; i < iters; ++i) {
#pragma unroll
        for (int c = 0; c < NCH; ++c) asm volatile("sin.approx.ftz.f32 %0, %0;" : "+f"(x[c]));
    }
    float s = 0.0f;
#pragma unroll
    for (int c = 0; c < NCH; ++c) s += x[c];
    sink[blockIdx.x * (int64_t)blockDim.x + threadIdx.x] = s;
}

}  // namespace
}  // namespace msgb

using namespace msgb;

extern "C" double msgb_peak_probe_ops(int kind, int64_t iters, int blocks, int threads) {
    const double lanes = (double)blocks * threads * (double)iters * NCH;
    switch (kind) {
        case MSGB_PEAK_FP32: return 2.0 * lanes;
        case MSGB_PEAK_FP32X2: return 4.0 * lanes;
        case MSGB_PEAK_FP64: return 2.0 * lanes;
        case MSGB_PEAK_MUFU: return lanes;
        default: return 0.0;
    }
}

extern "C" int msgb_peak_probe(int kind, int64_t iters, int blocks, int threads, float *sink,
                               msgb_stream_t stream) {
    if (iters < 1 || blocks < 1 || threads < 32 || threads > 1024 || (threads & 31))
        return fail(MSGB_ERR_ARG, "msgb_peak_probe: iters >= 1, blocks >= 1, threads a multiple of 32 in [32, 1024]");
    if (!sink) return fail(MSGB_ERR_ARG, "msgb_peak_probe: sink is NULL");
    cudaStream_t st = as_stream(stream);
    // a = 1 - 2^-20 and b small keep every chain finite and away from denormals
    switch (kind) {
        case MSGB_PEAK_FP32: peak_ffma_kernel<<<blocks, threads, 0, st>>>(iters, 0.99999905f, 1e-6f, sink); break;
        case MSGB_PEAK_FP32X2: peak_ffma2_kernel<<<blocks, threads, 0, st>>>(iters, 0.99999905f, 1e-6f, sink); break;
        case MSGB_PEAK_FP64: peak_dfma_kernel<<<blocks, threads, 0, st>>>(iters, 0.99999905, 1e-6, sink); break;
        case MSGB_PEAK_MUFU: peak_mufu_kernel<<<blocks, threads, 0, st>>>(iters, sink); break;
        default: return fail(MSGB_ERR_ARG, "msgb_peak_probe: unknown kind %d", kind);
    }
    return check_launch("msgb_peak_probe");
}
