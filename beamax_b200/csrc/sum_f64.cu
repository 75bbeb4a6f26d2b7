// Dense FP64 Gaussian-beam summation and its exact transpose.
//
// Forward: restates compute_gaussian_beam_real (beamax gb/core.py:194-329)
// with solve_hom_diag (gb/gb_solvers.py:356-422) fused in: every beam is
// evaluated at every (time, sensor) pair, as the reference does; there is no
// cutoff.  Each CTA owns a tile of TT times x TS sensors, keeps its outputs in
// registers and streams all 2n beams through shared memory, so every output is
// written exactly once and the summation order is fixed (deterministic).
//
// Transpose: one CTA per selected coefficient gathers
//   g_j = sum_{mode, t, s} 2 d(t, s) conj(A_j(t)) exp(-i w phi) exp(-w chi)
// over all times and sensors in a fixed order (no atomics).
#include "common.cuh"

namespace msgb {
namespace {

constexpr int TS = 64;          // sensors per tile
constexpr int TT = 16;          // times per tile
constexpr int THREADS = 256;
constexpr int BC = THREADS / TT;  // beams per shared-memory chunk
constexpr int TPT = TT / (THREADS / TS);  // times per thread

template <int D>
struct Rec64 {
    double x[D];
    double wp[D];
    double qr[D * (D + 1) / 2];  // w/2 * Re M (off-diagonals doubled)
    double qi[D * (D + 1) / 2];  // w/2 * Im M (off-diagonals doubled)
    double amp, ang;
};

template <int D>
__device__ __forceinline__ void load_beam(const BeamArgs &B, int64_t j, double *x0, double *p0,
                                          cd *al, cd &a0, double &w) {
#pragma unroll
    for (int i = 0; i < D; ++i) {
        x0[i] = B.x0[j * D + i];
        p0[i] = B.p0[j * D + i];
        al[i] = cd{B.alpha[2 * (j * D + i)], B.alpha[2 * (j * D + i) + 1]};
    }
    a0 = cd{B.a0[2 * j], B.a0[2 * j + 1]};
    w = B.omega[j];
}

template <int D>
__device__ __forceinline__ void make_rec(const ProbArgs &P, const BeamArgs &B, int64_t b, double t,
                                         Rec64<D> &r) {
    const int64_t j = b < B.n ? b : b - B.n;
    const double c0 = b < B.n ? P.c : -P.c;
    double x0[D], p0[D], w;
    cd al[D], a0;
    load_beam<D>(B, j, x0, p0, al, a0, w);
    HomState<D> st;
    hom_state<D>(x0, p0, al, a0, c0, t, st);
#pragma unroll
    for (int i = 0; i < D; ++i) {
        r.x[i] = P.periodic[i] ? pymod(st.x[i], P.L[i]) : st.x[i];
        r.wp[i] = w * p0[i];
    }
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
        for (int k = i; k < D; ++k) {
            const int q = sym_index<D>(i, k);
            const double f = (i == k ? 0.5 : 1.0) * w;
            r.qr[q] = f * st.M[q].re;
            r.qi[q] = f * st.M[q].im;
        }
    r.amp = 2.0 * hypot(st.A.re, st.A.im);
    r.ang = safe_angle(st.A);
}

template <int D>
__device__ __forceinline__ void eval_terms(const Rec64<D> &r, const double *s, const ProbArgs &P,
                                           bool any_periodic, double &ph, double &chi) {
    double Dl[D];
#pragma unroll
    for (int i = 0; i < D; ++i) {
        double di = s[i] - r.x[i];
        if (any_periodic && P.periodic[i]) di = di - P.L[i] * nearbyint(di / P.L[i]);
        Dl[i] = di;
    }
    double lin = 0.0, qr = 0.0, qi = 0.0;
#pragma unroll
    for (int i = 0; i < D; ++i) lin = fma(r.wp[i], Dl[i], lin);
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
        for (int k = i; k < D; ++k) {
            const int q = sym_index<D>(i, k);
            const double dd = Dl[i] * Dl[k];
            qr = fma(r.qr[q], dd, qr);
            qi = fma(r.qi[q], dd, qi);
        }
    ph = lin + qr + r.ang;
    chi = qi;
}

template <int D>
__global__ void __launch_bounds__(THREADS) fwd64_kernel(ProbArgs P, BeamArgs B, double *out) {
    __shared__ Rec64<D> recs[BC * TT];
    const int tid = threadIdx.x;
    const int sl = tid % TS;
    const int tg = tid / TS;
    const int64_t s_idx = (int64_t)blockIdx.x * TS + sl;
    const int64_t t_base = (int64_t)blockIdx.y * TT;
    const bool s_ok = s_idx < P.ns;
    bool any_periodic = false;
#pragma unroll
    for (int i = 0; i < D; ++i) any_periodic |= (P.periodic[i] != 0);

    double s[D];
#pragma unroll
    for (int i = 0; i < D; ++i) s[i] = s_ok ? P.sensors[s_idx * D + i] : 0.0;
    double acc[TPT];
#pragma unroll
    for (int k = 0; k < TPT; ++k) acc[k] = 0.0;

    const int64_t nb = B.modes == 1 ? B.n : 2 * B.n;        // end of the summed beams
    const int64_t b_lo = B.modes == 2 ? B.n : 0;             // start
    for (int64_t b0 = b_lo; b0 < nb; b0 += BC) {
        {
            const int bl = tid / TT, tl = tid % TT;
            const int64_t b = b0 + bl;
            const int64_t t = t_base + tl;
            Rec64<D> &r = recs[tid];
            if (b < nb && t < P.nt) {
                make_rec<D>(P, B, b, P.ts[t], r);
            } else {
                r.amp = 0.0;  // contributes exactly zero
#pragma unroll
                for (int i = 0; i < D; ++i) r.x[i] = 0.0, r.wp[i] = 0.0;
#pragma unroll
                for (int q = 0; q < D * (D + 1) / 2; ++q) r.qr[q] = 0.0, r.qi[q] = 0.0;
                r.ang = 0.0;
            }
        }
        __syncthreads();
        const int nbl = (nb - b0) < BC ? (int)(nb - b0) : BC;
        for (int bl = 0; bl < nbl; ++bl) {
#pragma unroll
            for (int k = 0; k < TPT; ++k) {
                const Rec64<D> &r = recs[bl * TT + tg + k * (THREADS / TS)];
                double ph, chi;
                eval_terms<D>(r, s, P, any_periodic, ph, chi);
                acc[k] += r.amp * cos(ph) * exp(-chi);
            }
        }
        __syncthreads();
    }
    if (s_ok) {
#pragma unroll
        for (int k = 0; k < TPT; ++k) {
            const int64_t t = t_base + tg + k * (THREADS / TS);
            if (t < P.nt) out[t * P.ns + s_idx] = acc[k];
        }
    }
}

template <int D>
__global__ void __launch_bounds__(THREADS) adj64_kernel(ProbArgs P, BeamArgs B, const double *data,
                                                        double *g) {
    const int64_t j = blockIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    bool any_periodic = false;
#pragma unroll
    for (int i = 0; i < D; ++i) any_periodic |= (P.periodic[i] != 0);
    double x0[D], p0[D], w;
    cd al[D], a0;
    load_beam<D>(B, j, x0, p0, al, a0, w);
    double acc_re = 0.0, acc_im = 0.0;
    for (int m = 0; m < 2; ++m) {
        if (!mode_on(B.modes, m)) continue;
        const double c0 = m == 0 ? P.c : -P.c;
        for (int64_t t = warp; t < P.nt; t += THREADS / 32) {
            HomState<D> st;
            hom_state<D>(x0, p0, al, a0, c0, P.ts[t], st);
            Rec64<D> r;
#pragma unroll
            for (int i = 0; i < D; ++i) {
                r.x[i] = P.periodic[i] ? pymod(st.x[i], P.L[i]) : st.x[i];
                r.wp[i] = w * p0[i];
            }
#pragma unroll
            for (int i = 0; i < D; ++i)
#pragma unroll
                for (int k = i; k < D; ++k) {
                    const int q = sym_index<D>(i, k);
                    const double f = (i == k ? 0.5 : 1.0) * w;
                    r.qr[q] = f * st.M[q].re;
                    r.qi[q] = f * st.M[q].im;
                }
            r.ang = 0.0;
            double sr = 0.0, si = 0.0;
            const double *drow = data + t * P.ns;
            for (int64_t s = lane; s < P.ns; s += 32) {
                double sp[D];
#pragma unroll
                for (int i = 0; i < D; ++i) sp[i] = P.sensors[s * D + i];
                double ph, chi;
                eval_terms<D>(r, sp, P, any_periodic, ph, chi);
                double sn, cs;
                sincos(ph, &sn, &cs);
                const double e = drow[s] * exp(-chi);
                sr = fma(e, cs, sr);
                si = fma(-e, sn, si);
            }
            // 2 conj(A) * (sr + i si)
            acc_re += 2.0 * (st.A.re * sr + st.A.im * si);
            acc_im += 2.0 * (st.A.re * si - st.A.im * sr);
        }
    }
    // Fixed-order block reduction.
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        acc_re += __shfl_down_sync(0xffffffffu, acc_re, o);
        acc_im += __shfl_down_sync(0xffffffffu, acc_im, o);
    }
    __shared__ double red[2][THREADS / 32];
    if (lane == 0) red[0][warp] = acc_re, red[1][warp] = acc_im;
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int k = 0; k < THREADS / 32; ++k) a += red[0][k], b += red[1][k];
        g[2 * j] = a;
        g[2 * j + 1] = b;
    }
}

// ---- trajectory records (msgb_rk4_trajectories rec64 layout) -------------
template <int D>
struct TrajView {
    int64_t nb, b_first;
    const double *rec64;
};

template <int D>
__device__ __forceinline__ void make_rec_traj(const ProbArgs &P, const BeamArgs &B, const TrajView<D> &T, int64_t bl,
                                              int64_t k, Rec64<D> &r) {
    constexpr int NR = 2 * D + 2 * D * D + 2;
    const double *y = T.rec64 + (k * T.nb + bl) * NR;
    const int64_t b = T.b_first + bl;
    const int64_t j = b < B.n ? b : b - B.n;
    const double w = B.omega[j];
#pragma unroll
    for (int i = 0; i < D; ++i) {
        r.x[i] = P.periodic[i] ? pymod(y[i], P.L[i]) : y[i];
        r.wp[i] = w * y[D + i];
    }
    const double *M = y + 2 * D;
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
        for (int l = i; l < D; ++l) {
            const int q = sym_index<D>(i, l);
            const double mre = i == l ? M[2 * (i * D + i)] : M[2 * (i * D + l)] + M[2 * (l * D + i)];
            const double mim = i == l ? M[2 * (i * D + i) + 1] : M[2 * (i * D + l) + 1] + M[2 * (l * D + i) + 1];
            r.qr[q] = 0.5 * w * mre;
            r.qi[q] = 0.5 * w * mim;
        }
    const cd Au = cd{y[2 * D + 2 * D * D], y[2 * D + 2 * D * D + 1]};
    const cd A = cd{B.a0[2 * j], B.a0[2 * j + 1]} * Au;
    r.amp = 2.0 * hypot(A.re, A.im);
    r.ang = safe_angle(A);
}

template <int D>
__global__ void __launch_bounds__(THREADS) fwd64_traj_kernel(ProbArgs P, BeamArgs B, TrajView<D> T, double *out) {
    __shared__ Rec64<D> recs[BC * TT];
    const int tid = threadIdx.x;
    const int sl = tid % TS;
    const int tg = tid / TS;
    const int64_t s_idx = (int64_t)blockIdx.x * TS + sl;
    const int64_t t_base = (int64_t)blockIdx.y * TT;
    const bool s_ok = s_idx < P.ns;
    bool any_periodic = false;
#pragma unroll
    for (int i = 0; i < D; ++i) any_periodic |= (P.periodic[i] != 0);
    double s[D];
#pragma unroll
    for (int i = 0; i < D; ++i) s[i] = s_ok ? P.sensors[s_idx * D + i] : 0.0;
    double acc[TPT];
#pragma unroll
    for (int k = 0; k < TPT; ++k) acc[k] = 0.0;
    for (int64_t b0 = 0; b0 < T.nb; b0 += BC) {
        {
            const int bl = tid / TT, tl = tid % TT;
            const int64_t b = b0 + bl, t = t_base + tl;
            Rec64<D> &r = recs[tid];
            if (b < T.nb && t < P.nt) {
                make_rec_traj<D>(P, B, T, b, t, r);
            } else {
                r.amp = 0.0;
#pragma unroll
                for (int i = 0; i < D; ++i) r.x[i] = 0.0, r.wp[i] = 0.0;
#pragma unroll
                for (int q = 0; q < D * (D + 1) / 2; ++q) r.qr[q] = 0.0, r.qi[q] = 0.0;
                r.ang = 0.0;
            }
        }
        __syncthreads();
        const int nbl = (T.nb - b0) < BC ? (int)(T.nb - b0) : BC;
        for (int bl = 0; bl < nbl; ++bl) {
#pragma unroll
            for (int k = 0; k < TPT; ++k) {
                const Rec64<D> &r = recs[bl * TT + tg + k * (THREADS / TS)];
                double ph, chi;
                eval_terms<D>(r, s, P, any_periodic, ph, chi);
                acc[k] += r.amp * cos(ph) * exp(-chi);
            }
        }
        __syncthreads();
    }
    if (s_ok) {
#pragma unroll
        for (int k = 0; k < TPT; ++k) {
            const int64_t t = t_base + tg + k * (THREADS / TS);
            if (t < P.nt) out[t * P.ns + s_idx] += acc[k];
        }
    }
}

template <int D>
__global__ void __launch_bounds__(THREADS) adj64_traj_kernel(ProbArgs P, BeamArgs B, TrajView<D> T, const double *data,
                                                             double *g) {
    const int64_t bl = blockIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    bool any_periodic = false;
#pragma unroll
    for (int i = 0; i < D; ++i) any_periodic |= (P.periodic[i] != 0);
    double acc_re = 0.0, acc_im = 0.0;
    for (int64_t t = warp; t < P.nt; t += THREADS / 32) {
        Rec64<D> r;
        make_rec_traj<D>(P, B, T, bl, t, r);
        const double amp = r.amp, ang = r.ang;
        r.ang = 0.0;
        double sr = 0.0, si = 0.0;
        const double *drow = data + t * P.ns;
        for (int64_t s = lane; s < P.ns; s += 32) {
            double sp[D];
#pragma unroll
            for (int i = 0; i < D; ++i) sp[i] = P.sensors[s * D + i];
            double ph, chi;
            eval_terms<D>(r, sp, P, any_periodic, ph, chi);
            double sn, cs;
            sincos(ph, &sn, &cs);
            const double e = drow[s] * exp(-chi);
            sr = fma(e, cs, sr);
            si = fma(-e, sn, si);
        }
        // amp/2 exp(-i ang) (sr + i si) * 2 = amp (cos ang - i sin ang)(sr + i si)
        double sa, ca;
        sincos(ang, &sa, &ca);
        acc_re += amp * (ca * sr + sa * si);
        acc_im += amp * (ca * si - sa * sr);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        acc_re += __shfl_down_sync(0xffffffffu, acc_re, o);
        acc_im += __shfl_down_sync(0xffffffffu, acc_im, o);
    }
    __shared__ double red[2][THREADS / 32];
    if (lane == 0) red[0][warp] = acc_re, red[1][warp] = acc_im;
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int k = 0; k < THREADS / 32; ++k) a += red[0][k], b += red[1][k];
        g[2 * bl] = a;
        g[2 * bl + 1] = b;
    }
}

}  // namespace
}  // namespace msgb

using namespace msgb;

extern "C" int msgb_sum_fwd_f64(const msgb_problem *prob, const msgb_beam_set *beams, double *out,
                                msgb_stream_t stream) {
    if (int e = validate_problem(prob)) return e;
    if (int e = validate_beams(prob, beams)) return e;
    if (!out) return fail(MSGB_ERR_ARG, "msgb_sum_fwd_f64: out is NULL");
    if (prob->nt == 0 || prob->ns == 0) return MSGB_OK;
    ProbArgs P = to_args(prob);
    BeamArgs B = to_args(beams);
    dim3 grid((unsigned)((prob->ns + TS - 1) / TS), (unsigned)((prob->nt + TT - 1) / TT));
    if (grid.y > 65535u) return fail(MSGB_ERR_UNSUPPORTED, "msgb_sum_fwd_f64: nt too large");
    cudaStream_t st = as_stream(stream);
    switch (prob->ndim) {
        case 1: fwd64_kernel<1><<<grid, THREADS, 0, st>>>(P, B, out); break;
        case 2: fwd64_kernel<2><<<grid, THREADS, 0, st>>>(P, B, out); break;
        default: fwd64_kernel<3><<<grid, THREADS, 0, st>>>(P, B, out); break;
    }
    return check_launch("msgb_sum_fwd_f64");
}

extern "C" int msgb_adj_gather_f64(const msgb_problem *prob, const msgb_beam_set *beams,
                                   const double *data, double *g, msgb_stream_t stream) {
    if (int e = validate_problem(prob)) return e;
    if (int e = validate_beams(prob, beams)) return e;
    if (!data || !g) return fail(MSGB_ERR_ARG, "msgb_adj_gather_f64: NULL data or g");
    if (beams->n == 0) return MSGB_OK;
    if (beams->n > 0x7fffffffLL) return fail(MSGB_ERR_UNSUPPORTED, "msgb_adj_gather_f64: too many beams");
    ProbArgs P = to_args(prob);
    BeamArgs B = to_args(beams);
    cudaStream_t st = as_stream(stream);
    const unsigned grid = (unsigned)beams->n;
    switch (prob->ndim) {
        case 1: adj64_kernel<1><<<grid, THREADS, 0, st>>>(P, B, data, g); break;
        case 2: adj64_kernel<2><<<grid, THREADS, 0, st>>>(P, B, data, g); break;
        default: adj64_kernel<3><<<grid, THREADS, 0, st>>>(P, B, data, g); break;
    }
    return check_launch("msgb_adj_gather_f64");
}

static int check_traj(const msgb_beam_set *beams, const msgb_trajectories *t, bool need64) {
    if (!t) return fail(MSGB_ERR_ARG, "trajectories are NULL");
    if (need64 && !t->rec64) return fail(MSGB_ERR_ARG, "FP64 trajectory records are NULL");
    if (t->nb < 0 || t->b_first < 0 || t->b_first + t->nb > 2 * beams->n)
        return fail(MSGB_ERR_ARG, "trajectory beam range outside [0, 2n)");
    return MSGB_OK;
}

extern "C" int msgb_sum_fwd_f64_traj(const msgb_problem *prob, const msgb_beam_set *beams,
                                     const msgb_trajectories *traj, double *out, msgb_stream_t stream) {
    if (int e = validate_problem(prob)) return e;
    if (int e = validate_beams(prob, beams)) return e;
    if (int e = check_traj(beams, traj, true)) return e;
    if (!out) return fail(MSGB_ERR_ARG, "msgb_sum_fwd_f64_traj: out is NULL");
    if (prob->nt == 0 || prob->ns == 0 || traj->nb == 0) return MSGB_OK;
    dim3 grid((unsigned)((prob->ns + TS - 1) / TS), (unsigned)((prob->nt + TT - 1) / TT));
    if (grid.y > 65535u) return fail(MSGB_ERR_UNSUPPORTED, "nt too large");
    ProbArgs P = to_args(prob);
    BeamArgs B = to_args(beams);
    cudaStream_t st = as_stream(stream);
    switch (prob->ndim) {
        case 1: fwd64_traj_kernel<1><<<grid, THREADS, 0, st>>>(P, B, TrajView<1>{traj->nb, traj->b_first, traj->rec64}, out); break;
        case 2: fwd64_traj_kernel<2><<<grid, THREADS, 0, st>>>(P, B, TrajView<2>{traj->nb, traj->b_first, traj->rec64}, out); break;
        default: fwd64_traj_kernel<3><<<grid, THREADS, 0, st>>>(P, B, TrajView<3>{traj->nb, traj->b_first, traj->rec64}, out); break;
    }
    return check_launch("msgb_sum_fwd_f64_traj");
}

extern "C" int msgb_adj_gather_f64_traj(const msgb_problem *prob, const msgb_beam_set *beams,
                                        const msgb_trajectories *traj, const double *data, double *g,
                                        msgb_stream_t stream) {
    if (int e = validate_problem(prob)) return e;
    if (int e = validate_beams(prob, beams)) return e;
    if (int e = check_traj(beams, traj, true)) return e;
    if (!data || !g) return fail(MSGB_ERR_ARG, "msgb_adj_gather_f64_traj: NULL data or g");
    if (traj->nb == 0) return MSGB_OK;
    if (traj->nb > 0x7fffffffLL) return fail(MSGB_ERR_UNSUPPORTED, "too many beams in one chunk");
    ProbArgs P = to_args(prob);
    BeamArgs B = to_args(beams);
    cudaStream_t st = as_stream(stream);
    const unsigned grid = (unsigned)traj->nb;
    switch (prob->ndim) {
        case 1: adj64_traj_kernel<1><<<grid, THREADS, 0, st>>>(P, B, TrajView<1>{traj->nb, traj->b_first, traj->rec64}, data, g); break;
        case 2: adj64_traj_kernel<2><<<grid, THREADS, 0, st>>>(P, B, TrajView<2>{traj->nb, traj->b_first, traj->rec64}, data, g); break;
        default: adj64_traj_kernel<3><<<grid, THREADS, 0, st>>>(P, B, TrajView<3>{traj->nb, traj->b_first, traj->rec64}, data, g); break;
    }
    return check_launch("msgb_adj_gather_f64_traj");
}
