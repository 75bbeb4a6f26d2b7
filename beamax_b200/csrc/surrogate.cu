// Trajectory surrogate: the data path around the BF16 MLP that predicts beam
// states in a heterogeneous medium (the MLP itself runs in mlp.cu).
//
// No counterpart in the reference (beamax integrates every beam with
// diffrax, gb/gb_solvers.py:940-1014).  The prediction is a correction to
// the closed-form homogeneous solution at the launch speed c0 = c(x0)
// (gb/gb_solvers.py:356-422), with tau = t - ts[0], T = ts[nt-1] - ts[0],
// |p0| = np:
//   features  x0 / L, mode p0 / np, log10(w) - 3, log10(Im alpha) + 3, tau / T
//   targets   (x - x_hom) / (c0 T), (p - p0) / np,
//             (M^-1 - M_hom^-1) np / (c0 T)   (upper triangle, re then im),
//             log(A / A_hom)                  (re, im)
// with M_hom^-1 = M0^-1 + mode c0 tau (I / np - p0 p0^T / np^3) (the
// homogeneous Riccati flow is linear in M^-1) and A_hom the closed-form
// amplitude.  M^-1 stays bounded where M itself grows.
//
// msgb_surrogate_records turns standardised predictions back into trajectory
// records and decides per beam whether to accept them: the Hamiltonian
// invariant c(x)|p| = c0 np (G is homogeneous of degree 1 in p) must hold to
// `residual_tol` at every time, and the validated position error bound times
// w np (the phase error it implies) must stay below `phase_tol`.  Rejected
// beams get status 3 (residual) or 4 (phase) and are re-integrated by
// msgb_ode_trajectories with only_flagged set.
#include "traj.cuh"

namespace msgb {
namespace {

struct SurrIO {
    int64_t nb, b_first, nq_t;
    const int32_t *t_index;
    int ld;
};

template <int D>
struct SurrDims {
    static constexpr int S = D * (D + 1) / 2;
    static constexpr int IN = 3 * D + 2;
    static constexpr int OUT = 2 * D + 2 * S + 2;
};

// Beam b of the 2n (b >= n: mode -1) and its launch data.
template <int D>
struct Launch {
    double x0[D], p0[D], np, w, mode, c0;
    cd alpha[D];
};

template <int D>
__device__ void load_launch(const MediumArgs &med, const BeamArgs &B, int64_t b, Launch<D> &l) {
    const int64_t j = b < B.n ? b : b - B.n;
    l.mode = b < B.n ? 1.0 : -1.0;
    double n2 = 0.0;
#pragma unroll
    for (int i = 0; i < D; ++i) {
        l.x0[i] = B.x0[j * D + i];
        l.p0[i] = B.p0[j * D + i];
        l.alpha[i] = cd{B.alpha[2 * (j * D + i)], B.alpha[2 * (j * D + i) + 1]};
        n2 += l.p0[i] * l.p0[i];
    }
    l.np = sqrt(n2);
    l.w = B.omega[j];
    double g[D], H[D * D];
    speed_eval<D>(med, l.x0, l.c0, g, H);
}

// Homogeneous reference at tau: x_hom, M_hom^-1 (full), A_hom (A from 1).
template <int D>
__device__ void hom_ref(const Launch<D> &l, double tau, double *xh, cd (*Minv)[D], cd &Ah) {
    const double cs = l.mode * l.c0;
    const double np3 = l.np * l.np * l.np;
#pragma unroll
    for (int i = 0; i < D; ++i) {
        xh[i] = l.x0[i] + cs * tau * l.p0[i] / l.np;
#pragma unroll
        for (int k = 0; k < D; ++k) {
            const double g = (i == k ? 1.0 / l.np : 0.0) - l.p0[i] * l.p0[k] / np3;
            Minv[i][k] = cd{cs * tau * g, 0.0};
        }
        Minv[i][i] = Minv[i][i] + divc(cd{1.0, 0.0}, l.alpha[i]);
    }
    HomState<D> st;
    hom_state<D>(l.x0, l.p0, l.alpha, cd{1.0, 0.0}, cs, tau, st);
    Ah = st.A;
}

// Inverse of a complex D x D matrix (cofactors); false when singular.
template <int D>
__device__ bool inv_c(const cd (*A)[D], cd (*R)[D]) {
    if (D == 1) {
        if (A[0][0].re == 0.0 && A[0][0].im == 0.0) return false;
        R[0][0] = divc(cd{1.0, 0.0}, A[0][0]);
        return true;
    }
    if (D == 2) {
        const cd det = A[0][0] * A[1 % D][1 % D] - A[0][1 % D] * A[1 % D][0];
        if (det.re == 0.0 && det.im == 0.0) return false;
        const cd id = divc(cd{1.0, 0.0}, det);
        R[0][0] = A[1 % D][1 % D] * id;
        R[1 % D][1 % D] = A[0][0] * id;
        R[0][1 % D] = cd{0.0, 0.0} - A[0][1 % D] * id;
        R[1 % D][0] = cd{0.0, 0.0} - A[1 % D][0] * id;
        return true;
    }
    cd C[D][D];
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
        for (int k = 0; k < D; ++k) {
            const int i1 = (i + 1) % D, i2 = (i + 2) % D, k1 = (k + 1) % D, k2 = (k + 2) % D;
            C[i][k] = A[i1][k1] * A[i2][k2] - A[i1][k2] * A[i2][k1];
        }
    cd det = cd{0.0, 0.0};
#pragma unroll
    for (int k = 0; k < D; ++k) det = det + A[0][k] * C[0][k];
    if (det.re == 0.0 && det.im == 0.0) return false;
    const cd id = divc(cd{1.0, 0.0}, det);
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
        for (int k = 0; k < D; ++k) R[i][k] = C[k][i] * id;
    return true;
}

__device__ __forceinline__ cd logc(cd z) { return cd{log(hypot(z.re, z.im)), atan2(z.im, z.re)}; }
__device__ __forceinline__ cd expc(cd z) {
    const double e = exp(z.re);
    double s, c;
    sincos(z.im, &s, &c);
    return cd{e * c, e * s};
}

__device__ __forceinline__ uint16_t to_bf16(float v) {
    uint32_t u = __float_as_uint(v);
    if ((u & 0x7f800000u) == 0x7f800000u) return (uint16_t)((u >> 16) | ((u & 0xffffu) ? 0x40u : 0u));
    u += 0x7fffu + ((u >> 16) & 1u);  // round to nearest even
    return (uint16_t)(u >> 16);
}

template <int D>
__global__ void features_kernel(ProbArgs P, MediumArgs med, BeamArgs B, SurrIO io, uint16_t *X) {
    const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (q >= io.nq_t * io.nb) return;
    const int64_t kq = q / io.nb, bl = q - kq * io.nb;
    const int64_t k = io.t_index ? io.t_index[kq] : kq;
    Launch<D> l;
    load_launch<D>(med, B, io.b_first + bl, l);
    const double T = P.nt > 1 ? P.ts[P.nt - 1] - P.ts[0] : 1.0;
    float f[SurrDims<D>::IN];
    int c = 0;
#pragma unroll
    for (int i = 0; i < D; ++i) f[c++] = (float)(l.x0[i] / P.L[i]);
#pragma unroll
    for (int i = 0; i < D; ++i) f[c++] = (float)(l.mode * l.p0[i] / l.np);
    f[c++] = (float)(log10(l.w) - 3.0);
#pragma unroll
    for (int i = 0; i < D; ++i) f[c++] = (float)(log10(fmax(fabs(l.alpha[i].im), 1e-300)) + 3.0);
    f[c++] = (float)((P.ts[k] - P.ts[0]) / T);
    uint16_t *row = X + q * io.ld;
    for (int i = 0; i < io.ld; ++i) row[i] = i < SurrDims<D>::IN ? to_bf16(f[i]) : (uint16_t)0;
}

template <int D>
__global__ void targets_kernel(ProbArgs P, MediumArgs med, BeamArgs B, SurrIO io, const double *rec64, float *Y) {
    constexpr int S = SurrDims<D>::S;
    constexpr int NR64 = 2 * D + 2 * D * D + 2;
    const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (q >= io.nq_t * io.nb) return;
    const int64_t kq = q / io.nb, bl = q - kq * io.nb;
    const int64_t k = io.t_index ? io.t_index[kq] : kq;
    Launch<D> l;
    load_launch<D>(med, B, io.b_first + bl, l);
    const double T = P.nt > 1 ? P.ts[P.nt - 1] - P.ts[0] : 1.0;
    const double tau = P.ts[k] - P.ts[0];
    const double Lc = l.c0 * T;
    double xh[D];
    cd Mh[D][D], Ah;
    hom_ref<D>(l, tau, xh, Mh, Ah);
    const double *r = rec64 + (k * io.nb + bl) * NR64;
    cd M[D][D], Mi[D][D];
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
        for (int m = 0; m < D; ++m) M[i][m] = cd{r[2 * D + 2 * (i * D + m)], r[2 * D + 2 * (i * D + m) + 1]};
    const bool ok = inv_c<D>(M, Mi);
    const cd A = cd{r[NR64 - 2], r[NR64 - 1]};
    float y[SurrDims<D>::OUT];
    int c = 0;
#pragma unroll
    for (int i = 0; i < D; ++i) y[c++] = (float)((r[i] - xh[i]) / Lc);
#pragma unroll
    for (int i = 0; i < D; ++i) y[c++] = (float)((r[D + i] - l.p0[i]) / l.np);
    const double sc = l.np / Lc;
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
        for (int m = i; m < D; ++m) {
            const cd d = ok ? 0.5 * (Mi[i][m] + Mi[m][i]) - Mh[i][m] : cd{0.0, 0.0};
            y[2 * D + sym_index<D>(i, m)] = (float)(sc * d.re);
            y[2 * D + S + sym_index<D>(i, m)] = (float)(sc * d.im);
        }
    c = 2 * D + 2 * S;
    const cd la = logc(divc(A, Ah));
    y[c++] = (float)la.re;
    y[c++] = (float)la.im;
    float *row = Y + q * io.ld;
    for (int i = 0; i < io.ld; ++i) row[i] = i < SurrDims<D>::OUT ? y[i] : 0.0f;
}

struct AcceptArgs {
    double residual_tol, phase_tol, pos_err;
};

template <int D>
__global__ void records_kernel(ProbArgs P, MediumArgs med, BeamArgs B, SurrIO io, const float *Yp, const float *mean,
                               const float *stdv, AcceptArgs acc, TrajArgs T, int tt_len) {
    constexpr int S = SurrDims<D>::S;
    const int64_t bl = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (bl >= io.nb) return;
    Launch<D> l;
    load_launch<D>(med, B, io.b_first + bl, l);
    const double Tt = P.nt > 1 ? P.ts[P.nt - 1] - P.ts[0] : 1.0;
    const double Lc = l.c0 * Tt;
    const double H0 = l.c0 * l.np;
    const int64_t ob = io.b_first - T.b_first + bl;  // index within the trajectory chunk
    RecordWriter<D> rw(P, T, ob, l.w, tt_len);
    double res = 0.0;
    bool finite = true;
    for (int64_t k = 0; k < P.nt; ++k) {
        const double tau = P.ts[k] - P.ts[0];
        double xh[D];
        cd Mh[D][D], Ah;
        hom_ref<D>(l, tau, xh, Mh, Ah);
        const float *row = Yp + (k * io.nb + bl) * io.ld;
        double y[SurrDims<D>::OUT];
#pragma unroll
        for (int i = 0; i < SurrDims<D>::OUT; ++i) y[i] = (double)row[i] * (double)stdv[i] + (double)mean[i];
        State<D> s;
#pragma unroll
        for (int i = 0; i < D; ++i) {
            s.x[i] = xh[i] + y[i] * Lc;
            s.p[i] = l.p0[i] + y[D + i] * l.np;
        }
        const double sc = Lc / l.np;
        cd Mi[D][D];
#pragma unroll
        for (int i = 0; i < D; ++i)
#pragma unroll
            for (int m = 0; m < D; ++m) {
                const int qq = sym_index<D>(i, m);
                Mi[i][m] = Mh[i][m] + cd{sc * y[2 * D + qq], sc * y[2 * D + S + qq]};
            }
        finite = finite && inv_c<D>(Mi, s.M);
        s.A = Ah * expc(cd{y[2 * D + 2 * S], y[2 * D + 2 * S + 1]});
        double c, g[D], Hs[D * D];
        speed_eval<D>(med, s.x, c, g, Hs);
        double n2 = 0.0;
#pragma unroll
        for (int i = 0; i < D; ++i) n2 += s.p[i] * s.p[i];
        const double r = fabs(c * sqrt(n2) / H0 - 1.0);
        res = isfinite(r) ? fmax(res, r) : 1e300;
        rw.put(k, s, false);
    }
    int code = 0;
    if (!finite || !(res <= acc.residual_tol))
        code = 3;
    else if (!(l.w * l.np * acc.pos_err <= acc.phase_tol))
        code = 4;
    if (T.status) T.status[ob] = code;
}

}  // namespace
}  // namespace msgb

using namespace msgb;

static int surr_common(const msgb_problem *prob, const msgb_medium *med, const msgb_beam_set *beams,
                       const msgb_surrogate_io *io, MediumArgs &M, SurrIO &S, int width) {
    if (int e = validate_problem(prob)) return e;
    if (int e = validate_beams(prob, beams)) return e;
    if (!io) return fail(MSGB_ERR_ARG, "surrogate io is NULL");
    if (int e = medium_args(prob, med, M)) return e;
    if (io->nb < 0 || io->b_first < 0 || io->b_first + io->nb > 2 * beams->n)
        return fail(MSGB_ERR_ARG, "beam range [%lld, %lld) outside [0, 2n)", (long long)io->b_first,
                    (long long)(io->b_first + io->nb));
    if (io->nq_t < 0) return fail(MSGB_ERR_ARG, "negative time count");
    if (io->ld < width)
        return fail(MSGB_ERR_ARG, "row stride %d below the %d columns this dimension needs", io->ld, width);
    S = SurrIO{io->nb, io->b_first, io->nq_t, io->t_index, io->ld};
    return MSGB_OK;
}

static int out_width(int d) { return d == 1 ? 6 : (d == 2 ? 12 : 20); }
static int in_width(int d) { return 3 * d + 2; }

extern "C" int msgb_surrogate_features(const msgb_problem *prob, const msgb_medium *med, const msgb_beam_set *beams,
                                       const msgb_surrogate_io *io, uint16_t *X, msgb_stream_t stream) {
    MediumArgs M;
    SurrIO S;
    if (int e = surr_common(prob, med, beams, io, M, S, prob ? in_width(prob->ndim) : 0)) return e;
    if (!X) return fail(MSGB_ERR_ARG, "msgb_surrogate_features: X is NULL");
    const int64_t n = S.nq_t * S.nb;
    if (n == 0) return MSGB_OK;
    const int blk = 128;
    const unsigned grid = (unsigned)((n + blk - 1) / blk);
    cudaStream_t st = as_stream(stream);
    ProbArgs P = to_args(prob);
    switch (prob->ndim) {
        case 1: features_kernel<1><<<grid, blk, 0, st>>>(P, M, to_args(beams), S, X); break;
        case 2: features_kernel<2><<<grid, blk, 0, st>>>(P, M, to_args(beams), S, X); break;
        default: features_kernel<3><<<grid, blk, 0, st>>>(P, M, to_args(beams), S, X); break;
    }
    return check_launch("msgb_surrogate_features");
}

extern "C" int msgb_surrogate_targets(const msgb_problem *prob, const msgb_medium *med, const msgb_beam_set *beams,
                                      const msgb_surrogate_io *io, const double *rec64, float *Y,
                                      msgb_stream_t stream) {
    MediumArgs M;
    SurrIO S;
    if (int e = surr_common(prob, med, beams, io, M, S, prob ? out_width(prob->ndim) : 0)) return e;
    if (!rec64 || !Y) return fail(MSGB_ERR_ARG, "msgb_surrogate_targets: NULL records or Y");
    const int64_t n = S.nq_t * S.nb;
    if (n == 0) return MSGB_OK;
    const int blk = 128;
    const unsigned grid = (unsigned)((n + blk - 1) / blk);
    cudaStream_t st = as_stream(stream);
    ProbArgs P = to_args(prob);
    switch (prob->ndim) {
        case 1: targets_kernel<1><<<grid, blk, 0, st>>>(P, M, to_args(beams), S, rec64, Y); break;
        case 2: targets_kernel<2><<<grid, blk, 0, st>>>(P, M, to_args(beams), S, rec64, Y); break;
        default: targets_kernel<3><<<grid, blk, 0, st>>>(P, M, to_args(beams), S, rec64, Y); break;
    }
    return check_launch("msgb_surrogate_targets");
}

extern "C" int msgb_surrogate_records(const msgb_problem *prob, const msgb_medium *med, const msgb_beam_set *beams,
                                      const msgb_surrogate_io *io, const float *Y, const float *mean,
                                      const float *stdv, const msgb_surrogate_accept *accept,
                                      const msgb_trajectories *out, msgb_stream_t stream) {
    MediumArgs M;
    SurrIO S;
    if (int e = surr_common(prob, med, beams, io, M, S, prob ? out_width(prob->ndim) : 0)) return e;
    if (!Y || !mean || !stdv || !accept || !out) return fail(MSGB_ERR_ARG, "msgb_surrogate_records: NULL argument");
    if (io->t_index || io->nq_t != prob->nt) return fail(MSGB_ERR_ARG, "records need predictions at every time");
    if (io->b_first < out->b_first || io->b_first + io->nb > out->b_first + out->nb)
        return fail(MSGB_ERR_ARG, "predicted beams lie outside the trajectory chunk");
    if (S.nb == 0 || prob->nt == 0) return MSGB_OK;
    if (out->pool) return fail(MSGB_ERR_UNSUPPORTED, "msgb_surrogate_records writes the dense FP32 layout (rec32)");
    AcceptArgs A{accept->residual_tol, accept->phase_tol, accept->pos_err};
    TrajArgs T{out->nb, out->b_first, beams->n, out->rec64, out->rec32, out->cull, out->status};
    const int blk = 64;
    const unsigned grid = (unsigned)((S.nb + blk - 1) / blk);
    cudaStream_t st = as_stream(stream);
    ProbArgs P = to_args(prob);
    switch (prob->ndim) {
        case 1: records_kernel<1><<<grid, blk, 0, st>>>(P, M, to_args(beams), S, Y, mean, stdv, A, T, MSGB_TIME_TILE); break;
        case 2: records_kernel<2><<<grid, blk, 0, st>>>(P, M, to_args(beams), S, Y, mean, stdv, A, T, MSGB_TIME_TILE); break;
        default: records_kernel<3><<<grid, blk, 0, st>>>(P, M, to_args(beams), S, Y, mean, stdv, A, T, MSGB_TIME_TILE); break;
    }
    return check_launch("msgb_surrogate_records");
}
