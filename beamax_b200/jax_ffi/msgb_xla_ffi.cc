// XLA FFI handlers over libmsgb's C ABI: the beam summation of the MSGB
// forward and its exact transpose as JAX custom calls on CUDA.
//
// Replaces the call of _compute_forward_result_jit in beamax's
// MSGBSolver.forward_with_params (solvers/msgb_solvers/msgb_solver.py:958-977)
// for the real sum methods: every selected coefficient j is propagated on
// both branches (modes +1 and -1, msgb_solver.py:612-619) and
//   out(t, s) = sum_j sum_mode 2 Re[a0_j K_{j,mode}(t, s)].
// The transpose handlers compute g_j = sum_{mode,t,s} 2 d(t, s) conj(K_{j,mode}).
//
// Written against the public XLA FFI API (xla/ffi/api/ffi.h, shipped in
// jaxlib's include directory, jax.ffi.include_dir()).  Buffers (device):
//   x0 (n, d) f64, p0 (n, d) f64, alpha (n, d) c128 (diagonal of M0),
//   a0 (n) c128, omega (n) f64, ts (nt) f64, sensors (ns, d) f64,
//   data (nt, ns) f64 / f32 for the transposes.
// Attributes: c (f64, constant sound speed), L (d f64, domain size),
//   periodic (d i64).
// The FP32 forward runs msgb_sum_fwd_f32_static (no scratch buffer needed);
// the FP32 transpose takes its workspace from XLA's scratch allocator.
#include <cuda_runtime.h>

#include <string>

#include "msgb.h"
#include "xla/ffi/api/ffi.h"

namespace ffi = xla::ffi;

namespace {

ffi::Error status(int rc, const char *what) {
    if (rc == MSGB_OK) return ffi::Error::Success();
    return ffi::Error(ffi::ErrorCode::kInternal, std::string(what) + ": " + msgb_last_error());
}

struct Geometry {
    msgb_problem prob{};
    msgb_beam_set beams{};
};

// Problem and beam descriptors from the buffers and attributes; returns an
// error for inconsistent shapes.
ffi::Error describe(ffi::Buffer<ffi::F64> x0, ffi::Buffer<ffi::F64> p0, ffi::Buffer<ffi::C128> alpha,
                    const void *a0, int64_t n_a0, ffi::Buffer<ffi::F64> omega, ffi::Buffer<ffi::F64> ts,
                    ffi::Buffer<ffi::F64> sensors, double c, ffi::Span<const double> L,
                    ffi::Span<const int64_t> periodic, Geometry &g) {
    const auto xd = x0.dimensions();
    if (xd.size() != 2) return ffi::Error(ffi::ErrorCode::kInvalidArgument, "x0 must be (n, d)");
    const int64_t n = xd[0], d = xd[1];
    if (d < 1 || d > 3 || (int64_t)L.size() != d || (int64_t)periodic.size() != d)
        return ffi::Error(ffi::ErrorCode::kInvalidArgument, "d must be 1..3 with L and periodic of length d");
    if (p0.element_count() != n * d || alpha.element_count() != n * d || n_a0 != n || omega.element_count() != n)
        return ffi::Error(ffi::ErrorCode::kInvalidArgument, "beam arrays disagree in n or d");
    const auto sd = sensors.dimensions();
    if (sd.size() != 2 || sd[1] != d) return ffi::Error(ffi::ErrorCode::kInvalidArgument, "sensors must be (ns, d)");
    g.prob.ndim = (int32_t)d;
    for (int a = 0; a < 3; ++a) {
        g.prob.periodic[a] = a < d ? (int32_t)(periodic[a] != 0) : 0;
        g.prob.L[a] = a < d ? L[a] : 1.0;
    }
    g.prob.c = c;
    g.prob.nt = ts.element_count();
    g.prob.ts = ts.typed_data();
    g.prob.ns = sd[0];
    g.prob.sensors = sensors.typed_data();
    g.beams.n = n;
    g.beams.x0 = x0.typed_data();
    g.beams.p0 = p0.typed_data();
    g.beams.alpha = reinterpret_cast<const double *>(alpha.typed_data());
    g.beams.a0 = reinterpret_cast<const double *>(a0);
    g.beams.omega = omega.typed_data();
    g.beams.modes = 0;
    return ffi::Error::Success();
}

ffi::Error SumFwdF64(cudaStream_t stream, ffi::Buffer<ffi::F64> x0, ffi::Buffer<ffi::F64> p0,
                     ffi::Buffer<ffi::C128> alpha, ffi::Buffer<ffi::C128> a0, ffi::Buffer<ffi::F64> omega,
                     ffi::Buffer<ffi::F64> ts, ffi::Buffer<ffi::F64> sensors, double c, ffi::Span<const double> L,
                     ffi::Span<const int64_t> periodic, ffi::ResultBuffer<ffi::F64> out) {
    Geometry g;
    if (auto e = describe(x0, p0, alpha, a0.typed_data(), a0.element_count(), omega, ts, sensors, c, L, periodic, g);
        e.failure())
        return e;
    return status(msgb_sum_fwd_f64(&g.prob, &g.beams, out->typed_data(), (msgb_stream_t)stream), "msgb_sum_fwd_f64");
}

ffi::Error SumFwdF32(cudaStream_t stream, ffi::Buffer<ffi::F64> x0, ffi::Buffer<ffi::F64> p0,
                     ffi::Buffer<ffi::C128> alpha, ffi::Buffer<ffi::C128> a0, ffi::Buffer<ffi::F64> omega,
                     ffi::Buffer<ffi::F64> ts, ffi::Buffer<ffi::F64> sensors, double c, ffi::Span<const double> L,
                     ffi::Span<const int64_t> periodic, double cutoff, ffi::ResultBuffer<ffi::F32> out) {
    Geometry g;
    if (auto e = describe(x0, p0, alpha, a0.typed_data(), a0.element_count(), omega, ts, sensors, c, L, periodic, g);
        e.failure())
        return e;
    msgb_sum_opts opts{};
    opts.cutoff = cutoff;
    return status(msgb_sum_fwd_f32_static(&g.prob, &g.beams, &opts, out->typed_data(), (msgb_stream_t)stream),
                  "msgb_sum_fwd_f32_static");
}

ffi::Error AdjF64(cudaStream_t stream, ffi::Buffer<ffi::F64> x0, ffi::Buffer<ffi::F64> p0, ffi::Buffer<ffi::C128> alpha,
                  ffi::Buffer<ffi::C128> a0_unit, ffi::Buffer<ffi::F64> omega, ffi::Buffer<ffi::F64> ts,
                  ffi::Buffer<ffi::F64> sensors, ffi::Buffer<ffi::F64> data, double c, ffi::Span<const double> L,
                  ffi::Span<const int64_t> periodic, ffi::ResultBuffer<ffi::C128> g_out) {
    Geometry g;
    if (auto e = describe(x0, p0, alpha, a0_unit.typed_data(), a0_unit.element_count(), omega, ts, sensors, c, L,
                          periodic, g);
        e.failure())
        return e;
    if (data.element_count() != g.prob.nt * g.prob.ns)
        return ffi::Error(ffi::ErrorCode::kInvalidArgument, "data must be (nt, ns)");
    return status(msgb_adj_gather_f64(&g.prob, &g.beams, data.typed_data(),
                                      reinterpret_cast<double *>(g_out->typed_data()), (msgb_stream_t)stream),
                  "msgb_adj_gather_f64");
}

ffi::Error AdjF32(cudaStream_t stream, ffi::ScratchAllocator scratch, ffi::Buffer<ffi::F64> x0,
                  ffi::Buffer<ffi::F64> p0, ffi::Buffer<ffi::C128> alpha, ffi::Buffer<ffi::C128> a0_unit,
                  ffi::Buffer<ffi::F64> omega, ffi::Buffer<ffi::F64> ts, ffi::Buffer<ffi::F64> sensors,
                  ffi::Buffer<ffi::F32> data, double c, ffi::Span<const double> L, ffi::Span<const int64_t> periodic,
                  double cutoff, ffi::ResultBuffer<ffi::C128> g_out) {
    Geometry g;
    if (auto e = describe(x0, p0, alpha, a0_unit.typed_data(), a0_unit.element_count(), omega, ts, sensors, c, L,
                          periodic, g);
        e.failure())
        return e;
    if (data.element_count() != g.prob.nt * g.prob.ns)
        return ffi::Error(ffi::ErrorCode::kInvalidArgument, "data must be (nt, ns)");
    const size_t bytes = msgb_sum_f32_workspace_size(&g.prob, g.beams.n);
    auto ws = scratch.Allocate(bytes, 256);
    if (!ws.has_value()) return ffi::Error(ffi::ErrorCode::kResourceExhausted, "msgb: scratch allocation failed");
    msgb_sum_opts opts{};
    opts.cutoff = cutoff;
    return status(msgb_adj_gather_f32(&g.prob, &g.beams, &opts, *ws, bytes, data.typed_data(),
                                      reinterpret_cast<double *>(g_out->typed_data()), (msgb_stream_t)stream),
                  "msgb_adj_gather_f32");
}

}  // namespace

#define MSGB_BEAM_ARGS                          \
    .Arg<ffi::Buffer<ffi::F64>>()  /* x0 */     \
        .Arg<ffi::Buffer<ffi::F64>>()  /* p0 */ \
        .Arg<ffi::Buffer<ffi::C128>>() /* alpha */ \
        .Arg<ffi::Buffer<ffi::C128>>() /* a0 */ \
        .Arg<ffi::Buffer<ffi::F64>>()  /* omega */ \
        .Arg<ffi::Buffer<ffi::F64>>()  /* ts */ \
        .Arg<ffi::Buffer<ffi::F64>>()  /* sensors */

XLA_FFI_DEFINE_HANDLER_SYMBOL(MsgbSumFwdF64, SumFwdF64,
                              ffi::Ffi::Bind()
                                  .Ctx<ffi::PlatformStream<cudaStream_t>>() MSGB_BEAM_ARGS
                                  .Attr<double>("c")
                                  .Attr<ffi::Span<const double>>("L")
                                  .Attr<ffi::Span<const int64_t>>("periodic")
                                  .Ret<ffi::Buffer<ffi::F64>>());

XLA_FFI_DEFINE_HANDLER_SYMBOL(MsgbSumFwdF32, SumFwdF32,
                              ffi::Ffi::Bind()
                                  .Ctx<ffi::PlatformStream<cudaStream_t>>() MSGB_BEAM_ARGS
                                  .Attr<double>("c")
                                  .Attr<ffi::Span<const double>>("L")
                                  .Attr<ffi::Span<const int64_t>>("periodic")
                                  .Attr<double>("cutoff")
                                  .Ret<ffi::Buffer<ffi::F32>>());

XLA_FFI_DEFINE_HANDLER_SYMBOL(MsgbAdjGatherF64, AdjF64,
                              ffi::Ffi::Bind()
                                  .Ctx<ffi::PlatformStream<cudaStream_t>>() MSGB_BEAM_ARGS
                                  .Arg<ffi::Buffer<ffi::F64>>()  /* data */
                                  .Attr<double>("c")
                                  .Attr<ffi::Span<const double>>("L")
                                  .Attr<ffi::Span<const int64_t>>("periodic")
                                  .Ret<ffi::Buffer<ffi::C128>>());

XLA_FFI_DEFINE_HANDLER_SYMBOL(MsgbAdjGatherF32, AdjF32,
                              ffi::Ffi::Bind()
                                  .Ctx<ffi::PlatformStream<cudaStream_t>>()
                                  .Ctx<ffi::ScratchAllocator>() MSGB_BEAM_ARGS
                                  .Arg<ffi::Buffer<ffi::F32>>()  /* data */
                                  .Attr<double>("c")
                                  .Attr<ffi::Span<const double>>("L")
                                  .Attr<ffi::Span<const int64_t>>("periodic")
                                  .Attr<double>("cutoff")
                                  .Ret<ffi::Buffer<ffi::C128>>());
