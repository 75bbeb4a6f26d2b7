// Boundary source of the principal-symbol adjoint and point evaluation of
// the sound speed.
//
// msgb_adjoint_source restates _form_adjoint_source (beamax
// solvers/msgb_solvers/msgb_solver.py:68-120): F = -c(x_s)^2 d_t(w r), the
// time derivative taken on the sampled Fourier grid, Re(ifft(2 pi i f
// fft(w r))) with f = fftfreq(nt, dt).  One batched 1D complex FFT per
// direction along the time axis (stride ns), cuFFT with the caller's work area.
#include <cufft.h>

#include "traj.cuh"

namespace msgb {
namespace {

__global__ void pack_kernel(const double *r, const double *w, int w_time_only, int64_t nt, int64_t ns,
                            double2 *z) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= nt * ns) return;
    double v = r[i];
    if (w) v *= w_time_only ? w[i / ns] : w[i];
    z[i] = make_double2(v, 0.0);
}

__global__ void derivative_kernel(double2 *z, int64_t nt, int64_t ns, double dt) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= nt * ns) return;
    const int64_t k = i / ns;
    // fftfreq: 0, 1, ..., ceil(nt/2) - 1, -floor(nt/2), ..., -1 over nt dt
    const int64_t kk = k < (nt + 1) / 2 ? k : k - nt;
    const double m = 2.0 * 3.141592653589793 * (double)kk / ((double)nt * dt) / (double)nt;  // with 1/nt of ifft
    const double2 v = z[i];
    z[i] = make_double2(-m * v.y, m * v.x);
}

__global__ void finish_kernel(const double2 *z, const double *c, int64_t nt, int64_t ns, double *out) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= nt * ns) return;
    const double cs = c[i % ns];
    out[i] = -(cs * cs) * z[i].x;
}

template <int D>
__global__ void speed_kernel(MediumArgs med, const double *x, int64_t n, double *c) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    double xi[D], g[D], H[D * D], ci;
#pragma unroll
    for (int a = 0; a < D; ++a) xi[a] = x[i * D + a];
    speed_eval<D>(med, xi, ci, g, H);
    c[i] = ci;
}

int make_time_plan(int64_t nt, int64_t ns, cufftHandle *h, size_t *work) {
    if (nt > 0x7fffffffLL || ns > 0x7fffffffLL) return fail(MSGB_ERR_UNSUPPORTED, "nt or ns too large for cuFFT");
    int n[1] = {(int)nt};
    int emb[1] = {(int)nt};
    cufftResult r = cufftCreate(h);
    if (r == CUFFT_SUCCESS) r = cufftSetAutoAllocation(*h, 0);
    if (r == CUFFT_SUCCESS)
        r = cufftMakePlanMany(*h, 1, n, emb, (int)ns, 1, emb, (int)ns, 1, CUFFT_Z2Z, (int)ns, work);
    if (r != CUFFT_SUCCESS) {
        cufftDestroy(*h);
        return fail(MSGB_ERR_CUDA, "adjoint source: cuFFT plan error %d", (int)r);
    }
    return MSGB_OK;
}

}  // namespace
}  // namespace msgb

using namespace msgb;

extern "C" size_t msgb_adjoint_source_workspace_size(int64_t nt, int64_t ns) {
    if (nt < 1 || ns < 1) return 0;
    cufftHandle h;
    size_t work = 0;
    if (make_time_plan(nt, ns, &h, &work)) return 0;
    cufftDestroy(h);
    return ((size_t)(nt * ns) * sizeof(double2) + 255) / 256 * 256 + work;
}

extern "C" int msgb_adjoint_source(const double *data, const double *window, int window_is_time_only, int64_t nt,
                                   int64_t ns, double dt, const double *c_at_sources, double *out, void *workspace,
                                   size_t workspace_bytes, msgb_stream_t stream) {
    if (!data || !c_at_sources || !out) return fail(MSGB_ERR_ARG, "msgb_adjoint_source: NULL argument");
    if (nt < 1 || ns < 1) return fail(MSGB_ERR_ARG, "nt and ns must be positive");
    if (!(dt > 0.0) || !isfinite(dt)) return fail(MSGB_ERR_ARG, "dt must be finite and positive");
    cufftHandle h;
    size_t work = 0;
    if (int e = make_time_plan(nt, ns, &h, &work)) return e;
    const size_t zb = ((size_t)(nt * ns) * sizeof(double2) + 255) / 256 * 256;
    if (!workspace || workspace_bytes < zb + work) {
        cufftDestroy(h);
        return fail(MSGB_ERR_WORKSPACE, "msgb_adjoint_source needs %zu workspace bytes", zb + work);
    }
    cudaStream_t st = as_stream(stream);
    double2 *z = (double2 *)workspace;
    const int64_t total = nt * ns;
    const int blk = 256;
    const unsigned grid = (unsigned)((total + blk - 1) / blk);
    pack_kernel<<<grid, blk, 0, st>>>(data, window, window_is_time_only, nt, ns, z);
    cufftResult r = cufftSetStream(h, st);
    if (r == CUFFT_SUCCESS) r = cufftSetWorkArea(h, (char *)workspace + zb);
    if (r == CUFFT_SUCCESS) r = cufftExecZ2Z(h, (cufftDoubleComplex *)z, (cufftDoubleComplex *)z, CUFFT_FORWARD);
    if (r == CUFFT_SUCCESS) derivative_kernel<<<grid, blk, 0, st>>>(z, nt, ns, dt);
    if (r == CUFFT_SUCCESS) r = cufftExecZ2Z(h, (cufftDoubleComplex *)z, (cufftDoubleComplex *)z, CUFFT_INVERSE);
    if (r == CUFFT_SUCCESS) finish_kernel<<<grid, blk, 0, st>>>(z, c_at_sources, nt, ns, out);
    cufftDestroy(h);
    if (r != CUFFT_SUCCESS) return fail(MSGB_ERR_CUDA, "msgb_adjoint_source: cuFFT error %d", (int)r);
    return check_launch("msgb_adjoint_source");
}

extern "C" int msgb_medium_speed(int32_t ndim, const msgb_medium *med, const double *x, int64_t n, double *c,
                                 msgb_stream_t stream) {
    if (ndim < 1 || ndim > 3) return fail(MSGB_ERR_ARG, "ndim must be 1, 2 or 3");
    if (n < 0) return fail(MSGB_ERR_ARG, "negative point count");
    if (n == 0) return MSGB_OK;
    if (!x || !c) return fail(MSGB_ERR_ARG, "msgb_medium_speed: NULL array");
    msgb_problem pr{};
    pr.ndim = ndim;
    MediumArgs M;
    if (int e = medium_args(&pr, med, M)) return e;
    const int blk = 128;
    const unsigned grid = (unsigned)((n + blk - 1) / blk);
    cudaStream_t st = as_stream(stream);
    switch (ndim) {
        case 1: speed_kernel<1><<<grid, blk, 0, st>>>(M, x, n, c); break;
        case 2: speed_kernel<2><<<grid, blk, 0, st>>>(M, x, n, c); break;
        default: speed_kernel<3><<<grid, blk, 0, st>>>(M, x, n, c); break;
    }
    return check_launch("msgb_medium_speed");
}
