// Heterogeneous beam propagation: FP64 integration of the ray, the complex
// Hessian (Riccati) and the amplitude, in a sound speed interpolated from a
// grid.
//
// Restates coupled_rhs_absorption (beamax gb/gb_solvers.py:820-867) and
// riccati_rhs (:787-817):
//   dx = G_p,  dp = -G_x,  dM = -(G_xx + G_xp M + M G_xp^T + M G_pp M),
//   dA = -A (c^2 tr M - G_x.G_p - G_p^T M G_p + lam G) / (2 G),
//   G = mode c(x) |p|,
// with c, grad c and hess c of make_c_function_from_grid (utils/interp.py:
// 31-263: n-linear or cubic B-spline tensor product, boundary maps
// nearest/wrap/reflect/mirror), evaluated with analytic weight derivatives.
// The reference integrates with adaptive Tsit5 under a PID step controller
// (:706-784).  Here: adaptive Dormand-Prince 5(4) with the same tolerances,
// error norm and step-count limit, or fixed-step RK4 (`substeps` equal steps
// per save interval).  One thread per beam; the state is written at every
// acquisition time.  A is integrated from 1 (the equation is linear in A):
// the summation multiplies by the beam amplitude.
#include <cstdlib>

#include "traj.cuh"

namespace msgb {
namespace {

template <int D>
__device__ void rhs(const MediumArgs &med, double mode, const State<D> &y, State<D> &dy) {
    double c, gc[D], hc[D * D];
    speed_eval<D>(med, y.x, c, gc, hc);
    double n2 = 0.0;
#pragma unroll
    for (int i = 0; i < D; ++i) n2 += y.p[i] * y.p[i];
    const double np = sqrt(n2);
    const double np3 = np * n2;
    const double G = mode * c * np;
    double Gx[D], Gp[D];
#pragma unroll
    for (int i = 0; i < D; ++i) {
        Gx[i] = mode * gc[i] * np;
        Gp[i] = mode * c * y.p[i] / np;
        dy.x[i] = Gp[i];
        dy.p[i] = -Gx[i];
    }
    double Gpp[D][D], Gxp[D][D];
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
        for (int k = 0; k < D; ++k) {
            Gpp[i][k] = mode * c * ((i == k ? 1.0 / np : 0.0) - y.p[i] * y.p[k] / np3);
            Gxp[i][k] = mode * gc[i] * y.p[k] / np;
        }
    // MGpp = M Gpp
    cd MG[D][D];
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
        for (int k = 0; k < D; ++k) {
            cd s = cd{0.0, 0.0};
#pragma unroll
            for (int l = 0; l < D; ++l) s = s + Gpp[l][k] * y.M[i][l];
            MG[i][k] = s;
        }
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
        for (int k = 0; k < D; ++k) {
            cd s = cd{mode * hc[i * D + k] * np, 0.0};
#pragma unroll
            for (int l = 0; l < D; ++l) {
                s = s + Gxp[i][l] * y.M[l][k];   // Gxp M
                s = s + Gxp[k][l] * y.M[i][l];   // M Gxp^T
                s = s + MG[i][l] * y.M[l][k];    // M Gpp M
            }
            dy.M[i][k] = cd{-s.re, -s.im};
        }
    cd trM = cd{0.0, 0.0};
    double gxgp = 0.0;
    cd gpmgp = cd{0.0, 0.0};
#pragma unroll
    for (int i = 0; i < D; ++i) {
        trM = trM + y.M[i][i];
        gxgp += Gx[i] * Gp[i];
#pragma unroll
        for (int k = 0; k < D; ++k) gpmgp = gpmgp + (Gp[i] * Gp[k]) * y.M[i][k];
    }
    cd num = (c * c) * trM;
    num = cd{num.re - gxgp - gpmgp.re + med.lam * G, num.im - gpmgp.im};
    const cd f = (-1.0 / (2.0 * G)) * num;
    dy.A = y.A * f;
}

template <int D>
__device__ __forceinline__ void axpy(State<D> &o, const State<D> &y, double h, const State<D> &k) {
#pragma unroll
    for (int i = 0; i < D; ++i) {
        o.x[i] = y.x[i] + h * k.x[i];
        o.p[i] = y.p[i] + h * k.p[i];
#pragma unroll
        for (int j = 0; j < D; ++j) o.M[i][j] = y.M[i][j] + h * k.M[i][j];
    }
    o.A = y.A + h * k.A;
}

// The adaptive integrator's state: M is complex symmetric, so only its upper
// triangle (sym_index order) is carried -- D(D+1)/2 entries instead of D^2,
// fewer registers per stage and fewer terms in the Riccati right-hand side.
template <int D>
struct SState {
    static constexpr int S = D * (D + 1) / 2;
    double x[D], p[D];
    cd M[S];
    cd A;
};

template <int D>
__device__ __forceinline__ void to_full(const SState<D> &s, State<D> &f) {
#pragma unroll
    for (int i = 0; i < D; ++i) {
        f.x[i] = s.x[i];
        f.p[i] = s.p[i];
#pragma unroll
        for (int k = 0; k < D; ++k) f.M[i][k] = s.M[sym_index<D>(i, k)];
    }
    f.A = s.A;
}

template <int D>
__device__ __forceinline__ void from_full(const State<D> &f, SState<D> &s) {
#pragma unroll
    for (int i = 0; i < D; ++i) {
        s.x[i] = f.x[i];
        s.p[i] = f.p[i];
#pragma unroll
        for (int k = i; k < D; ++k) s.M[sym_index<D>(i, k)] = f.M[i][k];
    }
    s.A = f.A;
}

// coupled_rhs_absorption on the symmetric state (the same terms as rhs; dM
// is formed for i <= k only).
// (The reciprocals 1/|p| and 1/|p|^3 replace FP64 divisions.)
template <int D, int KIND, bool F32M = false>
__device__ void rhs_sym(const MediumArgs &med, double mode, const SState<D> &y, SState<D> &dy) {
    double c, gc[D], hc[D * D];
    if (F32M && KIND != MSGB_MEDIUM_CONSTANT)
        speed_eval_f32<D, KIND>(med, y.x, c, gc, hc);
    else
        speed_eval_k<D, KIND>(med, y.x, c, gc, hc);
    double n2 = 0.0;
#pragma unroll
    for (int i = 0; i < D; ++i) n2 += y.p[i] * y.p[i];
    // FP32 path: 1/|p| from the FP64 reciprocal square root (one rounding
    // step from sqrt then divide, at a fraction of their instructions)
    const double inp = F32M ? rsqrt(n2) : 1.0 / sqrt(n2);
    const double np = F32M ? n2 * inp : sqrt(n2);
    const double inp3 = inp * inp * inp;
    const double G = mode * c * np;
    double Gx[D], Gp[D];
#pragma unroll
    for (int i = 0; i < D; ++i) {
        Gx[i] = mode * gc[i] * np;
        Gp[i] = mode * c * y.p[i] * inp;
        dy.x[i] = Gp[i];
        dy.p[i] = -Gx[i];
    }
    double Gpp[D][D], Gxp[D][D];
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
        for (int k = 0; k < D; ++k) {
            Gpp[i][k] = mode * c * ((i == k ? inp : 0.0) - y.p[i] * y.p[k] * inp3);
            Gxp[i][k] = mode * gc[i] * y.p[k] * inp;
        }
    cd MG[D][D];
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
        for (int k = 0; k < D; ++k) {
            cd sacc = cd{0.0, 0.0};
#pragma unroll
            for (int l = 0; l < D; ++l) sacc = sacc + Gpp[l][k] * y.M[sym_index<D>(i, l)];
            MG[i][k] = sacc;
        }
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
        for (int k = i; k < D; ++k) {
            cd sacc = cd{mode * hc[i * D + k] * np, 0.0};
#pragma unroll
            for (int l = 0; l < D; ++l) {
                sacc = sacc + Gxp[i][l] * y.M[sym_index<D>(l, k)];
                sacc = sacc + Gxp[k][l] * y.M[sym_index<D>(i, l)];
                sacc = sacc + MG[i][l] * y.M[sym_index<D>(l, k)];
            }
            dy.M[sym_index<D>(i, k)] = cd{-sacc.re, -sacc.im};
        }
    cd trM = cd{0.0, 0.0};
    double gxgp = 0.0;
    cd gpmgp = cd{0.0, 0.0};
#pragma unroll
    for (int i = 0; i < D; ++i) {
        trM = trM + y.M[sym_index<D>(i, i)];
        gxgp += Gx[i] * Gp[i];
#pragma unroll
        for (int k = 0; k < D; ++k) gpmgp = gpmgp + (Gp[i] * Gp[k]) * y.M[sym_index<D>(i, k)];
    }
    cd num = (c * c) * trM;
    num = cd{num.re - gxgp - gpmgp.re + med.lam * G, num.im - gpmgp.im};
    // -1 / (2 G) = -mode / (2 c |p|); the FP32 path takes 1/c in FP32 (the
    // amplitude's rate to FP32 precision, as its medium evaluation)
    const double ig = F32M ? -0.5 * mode * inp * (double)__frcp_rn((float)c) : -1.0 / (2.0 * G);
    const cd f = ig * num;
    dy.A = y.A * f;
}

template <int D>
__device__ void rk4_step(const MediumArgs &med, double mode, State<D> &y, double h) {
    State<D> k1, k2, k3, k4, t;
    rhs<D>(med, mode, y, k1);
    axpy<D>(t, y, 0.5 * h, k1);
    rhs<D>(med, mode, t, k2);
    axpy<D>(t, y, 0.5 * h, k2);
    rhs<D>(med, mode, t, k3);
    axpy<D>(t, y, h, k3);
    rhs<D>(med, mode, t, k4);
    const double h6 = h / 6.0;
#pragma unroll
    for (int i = 0; i < D; ++i) {
        y.x[i] += h6 * (k1.x[i] + 2.0 * k2.x[i] + 2.0 * k3.x[i] + k4.x[i]);
        y.p[i] += h6 * (k1.p[i] + 2.0 * k2.p[i] + 2.0 * k3.p[i] + k4.p[i]);
#pragma unroll
        for (int j = 0; j < D; ++j)
            y.M[i][j] = y.M[i][j] + h6 * (k1.M[i][j] + 2.0 * k2.M[i][j] + 2.0 * k3.M[i][j] + k4.M[i][j]);
    }
    y.A = y.A + h6 * (k1.A + 2.0 * k2.A + 2.0 * k3.A + k4.A);
}

// Dormand & Prince (1980) 5(4) pair.  Row s of DP_A gives stage s's input
// y + h sum_j DP_A[s][j] k_j; the last row equals the 5th-order weights
// (first same as last: k_7 = f(y_next) starts the next step).  DP_E = 5th- minus
// 4th-order weights, the local error estimate.
__constant__ double DP_A[7][6] = {
    {0, 0, 0, 0, 0, 0},
    {1.0 / 5, 0, 0, 0, 0, 0},
    {3.0 / 40, 9.0 / 40, 0, 0, 0, 0},
    {44.0 / 45, -56.0 / 15, 32.0 / 9, 0, 0, 0},
    {19372.0 / 6561, -25360.0 / 2187, 64448.0 / 6561, -212.0 / 729, 0, 0},
    {9017.0 / 3168, -355.0 / 33, 46732.0 / 5247, 49.0 / 176, -5103.0 / 18656, 0},
    {35.0 / 384, 0, 500.0 / 1113, 125.0 / 192, -2187.0 / 6784, 11.0 / 84}};
__constant__ double DP_E[7] = {35.0 / 384 - 5179.0 / 57600,
                               0.0,
                               500.0 / 1113 - 7571.0 / 16695,
                               125.0 / 192 - 393.0 / 640,
                               -2187.0 / 6784 + 92097.0 / 339200,
                               11.0 / 84 - 187.0 / 2100,
                               -1.0 / 40};

struct OdeArgs {
    int method, substeps;
    double rtol, atol, dt0;
    int64_t max_steps;
    int only_flagged, dense_output;
    unsigned long long *step_count;  // optional: attempted steps are added to it
};

template <int D>
struct NV {
    static constexpr int value = 2 * D + 2 * D * D + 2;  // doubles in State<D>
};

template <int D>
struct NVS {
    static constexpr int value = 2 * D + 2 * SState<D>::S + 2;  // doubles in SState<D>
};

template <int D>
__device__ __forceinline__ double *vals(State<D> &s) { return reinterpret_cast<double *>(&s); }
template <int D>
__device__ __forceinline__ const double *vals(const State<D> &s) { return reinterpret_cast<const double *>(&s); }
template <int D>
__device__ __forceinline__ double *vals(SState<D> &s) { return reinterpret_cast<double *>(&s); }
template <int D>
__device__ __forceinline__ const double *vals(const SState<D> &s) { return reinterpret_cast<const double *>(&s); }

// Weight of entry e of the symmetric state in the error norm: an
// off-diagonal M entry stands for two entries of the full matrix.
template <int D>
__host__ __device__ constexpr double sym_weight(int e) {
    return (e < 2 * D || e >= 2 * D + SState<D>::S) ? 1.0
         : (D == 2 ? (e - 2 * D == 1 ? 2.0 : 1.0)
         : D == 3 ? ((e - 2 * D == 1 || e - 2 * D == 2 || e - 2 * D == 4) ? 2.0 : 1.0)
         : 1.0);
}

// Squared magnitude of complex entry e of the state (x and p entries are real).
template <int D>
__device__ __forceinline__ double entry_abs2(const double *v, int e) {
    if (e < 2 * D) return v[e] * v[e];
    const int q = 2 * D + 2 * (e - 2 * D);
    return fma(v[q], v[q], v[q + 1] * v[q + 1]);
}

// Continuous-extension weights (Shampine 1986, the dense output of Hairer,
// Norsett & Wanner's dopri5): 4th-order interpolant inside an accepted step.
__constant__ double DP_D[7] = {-12715105075.0 / 11282082432.0, 0.0, 87487479700.0 / 32700410799.0,
                               -10690763975.0 / 1880347072.0, 701980252875.0 / 199316789632.0,
                               -1453857185.0 / 822651844.0, 69997945.0 / 29380423.0};

// Adaptive integration of one beam from ts[0] to ts[nt-1], one attempted
// step per call of attempt(); a step accepted right after a rejection does
// not grow the next one.  Save times, by o.dense_output:
//   0: a step that would pass the next save time is shortened to end on it,
//      and the proposal it replaced is kept for the following step (every
//      step is at most one save interval long, which also keeps the explicit
//      method inside its stability region for strongly focusing beams);
//   1: steps follow the error control alone (only the last is shortened to
//      end at ts[nt-1]) and save times inside a step are read from the
//      continuous extension, as diffrax's SaveAt(ts) reads its interpolant.
extern __shared__ double dopri_stage_smem[];
// Dynamic shared memory of the integrator kernels: 7 stages per lane (43 KB
// for a block of 64 lanes in 2D, 72 KB in 3D).
template <int D>
constexpr size_t dopri_smem_bytes(int blk) {
    return (size_t)blk * 7 * NVS<D>::value * sizeof(double);
}
// The mixed-precision integrator's: 7 FP64 ray stages and 7 FP32 Hessian and
// amplitude stages per lane (28 KB per 64 lanes in 2D, 46.6 KB in 3D).
template <int D>
constexpr size_t dopri_mix_smem_bytes(int blk) {
    return (size_t)blk * 7 * (2 * D * sizeof(double) + (D * (D + 1) + 2) * sizeof(float));
}
constexpr int kMixBlocks = 6;  // default blocks per SM of the mixed-precision integrator (measured best at config 3)

// DENSE: save times may fall inside a step (msgb_ode_opts.dense_output);
// without it every step ends on a save time and the continuous extension is
// not compiled (it is what pushed the kernel past 255 registers).
template <int D, int KIND, bool F32M = false, bool DENSE = true>
struct DopriBeam {
    SState<D> y;   // f(y) (first same as last) is stage 0 in shared memory
    double t, h, mode;
    int64_t steps, k;
    bool rejected;
    int code;  // 0 running or done, 1 non-finite, 2 step budget exhausted
    double *ks;  // this lane's stages in shared memory: stage j, entry c at ks[(j N + c) kst]
    int kst;

    __device__ void init(const MediumArgs &med, const ProbArgs &P, const OdeArgs &o, double mode_) {
        mode = mode_;
        h = o.dt0 > 0.0 ? o.dt0 : (P.nt > 1 ? P.ts[1] - P.ts[0] : 0.0);
        t = P.ts[0];
        steps = 0;
        k = 1;
        rejected = false;
        code = 0;
        SState<D> f0;
        rhs_sym<D, KIND, F32M>(med, mode, y, f0);
        const double *fv = vals(f0);
#pragma unroll
        for (int c = 0; c < NVS<D>::value; ++c) ks[c * kst] = fv[c];
    }

    // One attempt; returns true when the beam is finished (all save times
    // written or the step budget exhausted).
    __device__ bool attempt(const MediumArgs &med, const ProbArgs &P, const OdeArgs &o, RecordWriter<D> &rw) {
        constexpr int N = NVS<D>::value;
        constexpr int NE = 2 * D + SState<D>::S + 1;  // complex entries carried
        constexpr int NE_FULL = 2 * D + D * D + 1;     // entries of the full state (the norm's count)
        static_assert(sizeof(SState<D>) == N * sizeof(double), "SState<D> must be a plain array of doubles");
        if (k >= P.nt) return true;
        // Ending steps on the save times adds up to nt - 1 steps that an
        // integrator reading an interpolant would not take; they do not count
        // against the budget.
        if (steps >= o.max_steps + (o.dense_output ? 0 : P.nt - 1)) {
            code = 2;
            return true;
        }
        const double t_last = P.ts[P.nt - 1];
        const double target = o.dense_output ? t_last : P.ts[k];
        double hh = h;
        bool last = false;
        if (t + hh >= target) {
            hh = target - t;
            last = true;
        }
        // Stages in shared memory, one runtime loop over them: the right-hand
        // side is compiled once and the stages hold no registers (measured
        // 34 % faster than seven register-resident stages, which spilled and
        // limited the kernel to 8 warps per SM).
        SState<D> yt;
        const double *yv = vals(y);
#pragma unroll 1
        for (int s = 1; s < 7; ++s) {
            double acc[N];
#pragma unroll
            for (int c = 0; c < N; ++c) acc[c] = 0.0;
#pragma unroll 1
            for (int j = 0; j < s; ++j) {
                const double a = DP_A[s][j];
                if (a != 0.0) {
#pragma unroll
                    for (int c = 0; c < N; ++c) acc[c] += a * ks[(j * N + c) * kst];
                }
            }
            double *tv = vals(yt);
#pragma unroll
            for (int c = 0; c < N; ++c) tv[c] = yv[c] + hh * acc[c];
            SState<D> kn;
            rhs_sym<D, KIND, F32M>(med, mode, yt, kn);
            const double *kv = vals(kn);
#pragma unroll
            for (int c = 0; c < N; ++c) ks[(s * N + c) * kst] = kv[c];
        }
#define KSV(j, c) ks[((j) * N + (c)) * kst]
        // yt now holds the 5th-order solution (stage 7's input).
        const double *nv = vals(yt);
        double err;
        {
            double ev[N];
#pragma unroll
            for (int c = 0; c < N; ++c) {
                double acc = 0.0;
                for (int j = 0; j < 7; ++j) acc += DP_E[j] * KSV(j, c);
                ev[c] = hh * acc;
            }
            // (|e| / (atol + rtol max(|y0|, |y1|)))^2 from squared magnitudes:
            // one square root per entry instead of three.  The FP32 path
            // forms the norm, a step-size heuristic, in FP32.
            if (F32M) {
                const float at = (float)o.atol, rt = (float)o.rtol;
                float s32 = 0.0f;
#pragma unroll
                for (int e = 0; e < NE; ++e) {
                    const float sc = fmaf(rt, sqrtf((float)fmax(entry_abs2<D>(yv, e), entry_abs2<D>(nv, e))), at);
                    s32 = fmaf((float)sym_weight<D>(e), __fdividef((float)entry_abs2<D>(ev, e), sc * sc), s32);
                }
                err = (double)sqrtf(s32 * (1.0f / NE_FULL));
            } else {
                double sum = 0.0;
#pragma unroll
                for (int e = 0; e < NE; ++e) {
                    const double sc = o.atol + o.rtol * sqrt(fmax(entry_abs2<D>(yv, e), entry_abs2<D>(nv, e)));
                    sum += sym_weight<D>(e) * (entry_abs2<D>(ev, e) / (sc * sc));
                }
                err = sqrt(sum / NE_FULL);
            }
        }
        ++steps;
        if (!isfinite(err)) {
            h = 0.2 * hh;
            rejected = true;
            return false;
        }
        const double gr = F32M ? (double)(0.9f * exp2f(-0.2f * log2f((float)err))) : 0.9 * pow(err, -0.2);
        double fac = err == 0.0 ? 10.0 : fmin(10.0, fmax(0.2, gr));
        if (err <= 1.0) {
            if (rejected) fac = fmin(fac, 1.0);
            rejected = false;
            const double t_new = last ? target : t + hh;
            while (k < P.nt && P.ts[k] <= t_new) {
                if (!DENSE || P.ts[k] == t_new) {
                    State<D> yf;
                    to_full(yt, yf);
                    rw.put(k, yf, false);
                } else {
                    const double th = (P.ts[k] - t) / hh;
                    SState<D> yd;
                    double *dv = vals(yd);
#pragma unroll
                    for (int c = 0; c < N; ++c) {
                        double r5 = 0.0;
                        for (int j = 0; j < 7; ++j) {
                            const double dj = DP_D[j];
                            if (dj != 0.0) r5 += dj * KSV(j, c);
                        }
                        r5 *= hh;
                        const double r2 = nv[c] - yv[c];
                        const double r3 = hh * KSV(0, c) - r2;
                        const double r4 = r2 - hh * KSV(6, c) - r3;
                        dv[c] = yv[c] + th * (r2 + (1.0 - th) * (r3 + th * (r4 + (1.0 - th) * r5)));
                    }
                    State<D> yf;
                    to_full(yd, yf);
                    rw.put(k, yf, false);
                }
                ++k;
            }
            t = t_new;
            y = yt;
#pragma unroll
            for (int c = 0; c < N; ++c) KSV(0, c) = KSV(6, c);  // first same as last
#undef KSV
            h = (last && !o.dense_output) ? fmax(hh * fac, h) : hh * fac;
        } else {
            h = hh * fmin(1.0, fac);
            rejected = true;
        }
        return k >= P.nt;
    }
};

// ---- the FP32 path's mixed-precision integrator ------------------------------
// The ray (x, p) stays FP64: the summation's phase w p.(s - x) needs it.  The
// Hessian M and the amplitude A, which enter the FP32 summation as FP32
// values, are integrated in FP32 with the same Dormand-Prince stages and the
// same error control (their FP32 rounding, ~1e-7 relative per step, stays far
// below the FP32 path's 1e-3 budget).  Half the FP64 dependency chains, 2/3 of
// the stage memory and fewer registers than DopriBeam.
template <int D>
struct MState {
    static constexpr int S = D * (D + 1) / 2;
    static constexpr int ND = 2 * D;      // doubles: x, p
    static constexpr int NF = 2 * S + 2;  // floats: M (re, im) in sym_index order, A (re, im)
    double r[ND];
    float f[NF];
};

template <int D>
__device__ __forceinline__ void mix_to_full(const MState<D> &s, State<D> &o) {
    constexpr int S = MState<D>::S;
#pragma unroll
    for (int i = 0; i < D; ++i) {
        o.x[i] = s.r[i];
        o.p[i] = s.r[D + i];
#pragma unroll
        for (int k = 0; k < D; ++k) {
            const int q = sym_index<D>(i, k);
            o.M[i][k] = cd{(double)s.f[2 * q], (double)s.f[2 * q + 1]};
        }
    }
    o.A = cd{(double)s.f[2 * S], (double)s.f[2 * S + 1]};
}

template <int D>
__device__ __forceinline__ void mix_from_full(const State<D> &o, MState<D> &s) {
    constexpr int S = MState<D>::S;
#pragma unroll
    for (int i = 0; i < D; ++i) {
        s.r[i] = o.x[i];
        s.r[D + i] = o.p[i];
#pragma unroll
        for (int k = i; k < D; ++k) {
            const int q = sym_index<D>(i, k);
            s.f[2 * q] = (float)o.M[i][k].re;
            s.f[2 * q + 1] = (float)o.M[i][k].im;
        }
    }
    s.f[2 * S] = (float)o.A.re;
    s.f[2 * S + 1] = (float)o.A.im;
}

// coupled_rhs_absorption: the ray terms in FP64, the Riccati and amplitude
// terms in FP32 (the same terms as rhs_sym).
template <int D, int KIND>
__device__ void rhs_mix(const MediumArgs &med, double mode, const MState<D> &y, MState<D> &dy) {
    constexpr int S = MState<D>::S;
    double c, gc[D], hc[D * D];
    if (KIND != MSGB_MEDIUM_CONSTANT)
        speed_eval_f32<D, KIND>(med, y.r, c, gc, hc);
    else
        speed_eval_k<D, KIND>(med, y.r, c, gc, hc);
    const double *p = y.r + D;
    double n2 = 0.0;
#pragma unroll
    for (int i = 0; i < D; ++i) n2 += p[i] * p[i];
    const double inp = rsqrt(n2);
    const double np = n2 * inp;
    const double mc_inp = mode * c * inp, mnp = mode * np;
#pragma unroll
    for (int i = 0; i < D; ++i) {
        dy.r[i] = mc_inp * p[i];     // G_p
        dy.r[D + i] = -mnp * gc[i];  // -G_x
    }
    const float m = (float)mode, cf = (float)c, npf = (float)np, inpf = (float)inp;
    const float inp3 = inpf * inpf * inpf;
    float pf[D], Gx[D], Gp[D];
#pragma unroll
    for (int i = 0; i < D; ++i) {
        pf[i] = (float)p[i];
        Gp[i] = (float)dy.r[i];
        Gx[i] = -(float)dy.r[D + i];
    }
    float Gpp[D][D], Gxp[D][D];
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
        for (int k = 0; k < D; ++k) {
            Gpp[i][k] = m * cf * ((i == k ? inpf : 0.0f) - pf[i] * pf[k] * inp3);
            Gxp[i][k] = Gx[i] * pf[k] * inpf * inpf;  // m gc_i |p| p_k / |p|^2 = m gc_i p_k / |p|
        }
    auto Mre = [&](int i, int k) { return y.f[2 * sym_index<D>(i, k)]; };
    auto Mim = [&](int i, int k) { return y.f[2 * sym_index<D>(i, k) + 1]; };
    float MGr[D][D], MGi[D][D];
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
        for (int k = 0; k < D; ++k) {
            float sr = 0.0f, si = 0.0f;
#pragma unroll
            for (int l = 0; l < D; ++l) {
                sr = fmaf(Gpp[l][k], Mre(i, l), sr);
                si = fmaf(Gpp[l][k], Mim(i, l), si);
            }
            MGr[i][k] = sr;
            MGi[i][k] = si;
        }
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
        for (int k = i; k < D; ++k) {
            float sr = m * (float)hc[i * D + k] * npf, si = 0.0f;
#pragma unroll
            for (int l = 0; l < D; ++l) {
                sr = fmaf(Gxp[i][l], Mre(l, k), sr);
                si = fmaf(Gxp[i][l], Mim(l, k), si);
                sr = fmaf(Gxp[k][l], Mre(i, l), sr);
                si = fmaf(Gxp[k][l], Mim(i, l), si);
                // (MG)_il M_lk, complex
                sr = fmaf(MGr[i][l], Mre(l, k), fmaf(-MGi[i][l], Mim(l, k), sr));
                si = fmaf(MGr[i][l], Mim(l, k), fmaf(MGi[i][l], Mre(l, k), si));
            }
            const int q = sym_index<D>(i, k);
            dy.f[2 * q] = -sr;
            dy.f[2 * q + 1] = -si;
        }
    float trr = 0.0f, tri = 0.0f, gxgp = 0.0f, gmr = 0.0f, gmi = 0.0f;
#pragma unroll
    for (int i = 0; i < D; ++i) {
        trr += Mre(i, i);
        tri += Mim(i, i);
        gxgp = fmaf(Gx[i], Gp[i], gxgp);
#pragma unroll
        for (int k = 0; k < D; ++k) {
            const float gg = Gp[i] * Gp[k];
            gmr = fmaf(gg, Mre(i, k), gmr);
            gmi = fmaf(gg, Mim(i, k), gmi);
        }
    }
    const float c2 = cf * cf;
    const float nr = fmaf(c2, trr, -gxgp) - gmr + (float)med.lam * (m * cf * npf);
    const float ni = fmaf(c2, tri, -gmi);
    // -1 / (2 G) = -mode / (2 c |p|)
    const float ig = -0.5f * m * inpf * __frcp_rn(cf);
    const float fr = ig * nr, fi = ig * ni;
    const float ar = y.f[2 * S], ai = y.f[2 * S + 1];
    dy.f[2 * S] = fmaf(ar, fr, -ai * fi);
    dy.f[2 * S + 1] = fmaf(ar, fi, ai * fr);
}

__constant__ float DP_A32[7][6] = {
    {0, 0, 0, 0, 0, 0},
    {(float)(1.0 / 5), 0, 0, 0, 0, 0},
    {(float)(3.0 / 40), (float)(9.0 / 40), 0, 0, 0, 0},
    {(float)(44.0 / 45), (float)(-56.0 / 15), (float)(32.0 / 9), 0, 0, 0},
    {(float)(19372.0 / 6561), (float)(-25360.0 / 2187), (float)(64448.0 / 6561), (float)(-212.0 / 729), 0, 0},
    {(float)(9017.0 / 3168), (float)(-355.0 / 33), (float)(46732.0 / 5247), (float)(49.0 / 176),
     (float)(-5103.0 / 18656), 0},
    {(float)(35.0 / 384), 0, (float)(500.0 / 1113), (float)(125.0 / 192), (float)(-2187.0 / 6784), (float)(11.0 / 84)}};
__constant__ float DP_E32[7] = {(float)(35.0 / 384 - 5179.0 / 57600),
                                0.0f,
                                (float)(500.0 / 1113 - 7571.0 / 16695),
                                (float)(125.0 / 192 - 393.0 / 640),
                                (float)(-2187.0 / 6784 + 92097.0 / 339200),
                                (float)(11.0 / 84 - 187.0 / 2100),
                                (float)(-1.0 / 40)};

// DopriBeam's step (save times landed on, no continuous extension) on the
// mixed state.  Stages in shared memory: the FP64 ray stages, then the FP32
// Hessian and amplitude stages, each entry strided by the block size.
template <int D, int KIND>
struct DopriMix {
    static constexpr int ND = MState<D>::ND, NF = MState<D>::NF, S = MState<D>::S;
    MState<D> y;
    double t, h, mode;
    int64_t steps, k;
    bool rejected;
    int code;
    double *k64;  // stage j, entry c at k64[(j ND + c) kst]
    float *k32;   // stage j, entry c at k32[(j NF + c) kst]
    // the block size (every integrator launch has 64 lanes): a compile-time
    // stride turns the stage addresses into immediate offsets
    static constexpr int kst = 64;

    __device__ void init(const MediumArgs &med, const ProbArgs &P, const OdeArgs &o, double mode_) {
        mode = mode_;
        h = o.dt0 > 0.0 ? o.dt0 : (P.nt > 1 ? P.ts[1] - P.ts[0] : 0.0);
        t = P.ts[0];
        steps = 0;
        k = 1;
        rejected = false;
        code = 0;
        MState<D> f0;
        rhs_mix<D, KIND>(med, mode, y, f0);
#pragma unroll
        for (int c = 0; c < ND; ++c) k64[c * kst] = f0.r[c];
#pragma unroll
        for (int c = 0; c < NF; ++c) k32[c * kst] = f0.f[c];
    }

    __device__ bool attempt(const MediumArgs &med, const ProbArgs &P, const OdeArgs &o, RecordWriter<D> &rw) {
        constexpr int NE = 2 * D + S + 1;          // entries of the error norm (x, p real; M, A complex)
        constexpr int NE_FULL = 2 * D + D * D + 1;  // entries of the full state
        if (k >= P.nt) return true;
        if (steps >= o.max_steps + P.nt - 1) {
            code = 2;
            return true;
        }
        const double target = P.ts[k];
        double hh = h;
        bool last = false;
        if (t + hh >= target) {
            hh = target - t;
            last = true;
        }
        const float hf = (float)hh;
        MState<D> yt;
#pragma unroll 1
        for (int s = 1; s < 7; ++s) {
            double a64[ND];
            float a32[NF];
#pragma unroll
            for (int c = 0; c < ND; ++c) a64[c] = 0.0;
#pragma unroll
            for (int c = 0; c < NF; ++c) a32[c] = 0.0f;
#pragma unroll 1
            for (int j = 0; j < s; ++j) {
                const double a = DP_A[s][j];
                if (a != 0.0) {
                    const float af = DP_A32[s][j];
#pragma unroll
                    for (int c = 0; c < ND; ++c) a64[c] += a * k64[(j * ND + c) * kst];
#pragma unroll
                    for (int c = 0; c < NF; ++c) a32[c] = fmaf(af, k32[(j * NF + c) * kst], a32[c]);
                }
            }
#pragma unroll
            for (int c = 0; c < ND; ++c) yt.r[c] = y.r[c] + hh * a64[c];
#pragma unroll
            for (int c = 0; c < NF; ++c) yt.f[c] = fmaf(hf, a32[c], y.f[c]);
            MState<D> kn;
            rhs_mix<D, KIND>(med, mode, yt, kn);
#pragma unroll
            for (int c = 0; c < ND; ++c) k64[(s * ND + c) * kst] = kn.r[c];
#pragma unroll
            for (int c = 0; c < NF; ++c) k32[(s * NF + c) * kst] = kn.f[c];
        }
        // yt holds the 5th-order solution.  Error norm in FP32, as DopriBeam's
        // FP32-path variant forms it.
        float s32 = 0.0f;
        {
            const float at = (float)o.atol, rt = (float)o.rtol;
#pragma unroll
            for (int c = 0; c < ND; ++c) {
                double acc = 0.0;
                for (int j = 0; j < 7; ++j) acc += DP_E[j] * k64[(j * ND + c) * kst];
                const float e = (float)(hh * acc);
                const float sc = fmaf(rt, (float)fmax(fabs(y.r[c]), fabs(yt.r[c])), at);
                s32 = fmaf(e, __fdividef(e, sc * sc), s32);
            }
#pragma unroll
            for (int q = 0; q < S + 1; ++q) {
                float er = 0.0f, ei = 0.0f;
                for (int j = 0; j < 7; ++j) {
                    er = fmaf(DP_E32[j], k32[(j * NF + 2 * q) * kst], er);
                    ei = fmaf(DP_E32[j], k32[(j * NF + 2 * q + 1) * kst], ei);
                }
                er *= hf;
                ei *= hf;
                const float y0 = fmaf(y.f[2 * q], y.f[2 * q], y.f[2 * q + 1] * y.f[2 * q + 1]);
                const float y1 = fmaf(yt.f[2 * q], yt.f[2 * q], yt.f[2 * q + 1] * yt.f[2 * q + 1]);
                const float sc = fmaf(rt, sqrtf(fmaxf(y0, y1)), at);
                s32 = fmaf((float)sym_weight<D>(2 * D + q), __fdividef(fmaf(er, er, ei * ei), sc * sc), s32);
            }
        }
        const float err = sqrtf(s32 * (1.0f / NE_FULL));
        (void)NE;
        ++steps;
        if (!isfinite(err)) {
            h = 0.2 * hh;
            rejected = true;
            return false;
        }
        double fac = err == 0.0f ? 10.0 : fmin(10.0, fmax(0.2, (double)(0.9f * exp2f(-0.2f * log2f(err)))));
        if (err <= 1.0f) {
            if (rejected) fac = fmin(fac, 1.0);
            rejected = false;
            const double t_new = last ? target : t + hh;
            while (k < P.nt && P.ts[k] <= t_new) {
                State<D> yf;
                mix_to_full(yt, yf);
                rw.put(k, yf, false);
                ++k;
            }
            t = t_new;
            y = yt;
#pragma unroll
            for (int c = 0; c < ND; ++c) k64[c * kst] = k64[(6 * ND + c) * kst];  // first same as last
#pragma unroll
            for (int c = 0; c < NF; ++c) k32[c * kst] = k32[(6 * NF + c) * kst];
            h = last ? fmax(hh * fac, h) : hh * fac;
        } else {
            h = hh * fmin(1.0, fac);
            rejected = true;
        }
        return k >= P.nt;
    }
};

template <int D>
__device__ void launch_state(const BeamArgs &B, const TrajArgs &T, int64_t bl, State<D> &y, double &mode, double &w) {
    const int64_t b = T.b_first + bl;
    const int64_t j = b < B.n ? b : b - B.n;
    mode = b < B.n ? 1.0 : -1.0;
#pragma unroll
    for (int i = 0; i < D; ++i) {
        y.x[i] = B.x0[j * D + i];
        y.p[i] = B.p0[j * D + i];
#pragma unroll
        for (int k = 0; k < D; ++k) y.M[i][k] = cd{0.0, 0.0};
        y.M[i][i] = cd{B.alpha[2 * (j * D + i)], B.alpha[2 * (j * D + i) + 1]};
    }
    y.A = cd{1.0, 0.0};
    w = B.omega[j];
}

// Adaptive integration with persistent lanes: thread i integrates beams
// i, i + stride, i + 2 stride, ... one attempted step per loop trip, so a
// lane whose beam finishes early starts its next beam instead of idling
// until the slowest beam of its warp is done.
// MINB: resident 64-lane blocks per SM the register allocation is bounded for
// (the stages take 43 KB of shared memory per block in 2D, so at most 5 fit).
template <int D, int KIND, int MINB, bool F32M, bool DENSE>
__global__ void __launch_bounds__(64, MINB)
dopri_kernel(ProbArgs P, MediumArgs med, BeamArgs B, TrajArgs T, OdeArgs o, int tt_len) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int64_t bl = blockIdx.x * (int64_t)blockDim.x + threadIdx.x - stride;
    bool active = false;
    DopriBeam<D, KIND, F32M, DENSE> s;
    s.ks = dopri_stage_smem + threadIdx.x;
    s.kst = blockDim.x;
    RecordWriter<D> rw(P, T, 0, 0.0, tt_len);
    unsigned long long lane_steps = 0;
    for (;;) {
        if (!active) {
            bl += stride;
            while (bl < T.nb && o.only_flagged && T.status[bl] == 0) bl += stride;  // already accepted
            if (bl < T.nb) {
                double mode, w;
                State<D> y0;
                launch_state<D>(B, T, bl, y0, mode, w);
                from_full(y0, s.y);
                rw.reset(bl, w);
                rw.put(0, y0, false);
                s.init(med, P, o, mode);
                active = true;
            }
        }
        if (!__any_sync(0xffffffffu, active)) break;
        if (active && s.attempt(med, P, o, rw)) {
            bool fin = isfinite(s.y.A.re) && isfinite(s.y.A.im);
#pragma unroll
            for (int i = 0; i < D; ++i) fin = fin && isfinite(s.y.x[i]) && isfinite(s.y.p[i]);
            if (!fin && s.code == 0) s.code = 1;
            if (s.k < P.nt) {  // after a failure: the last state
                State<D> yf;
                to_full(s.y, yf);
                for (int64_t k = s.k; k < P.nt; ++k) rw.put(k, yf, true);
            }
            if (T.status) T.status[bl] = s.code;
            lane_steps += (unsigned long long)s.steps;
            active = false;
        }
    }
    if (o.step_count) {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) lane_steps += __shfl_xor_sync(0xffffffffu, lane_steps, off);
        if ((threadIdx.x & 31) == 0 && lane_steps) atomicAdd(o.step_count, lane_steps);
    }
}

// dopri_kernel with the FP32 path's mixed-precision state (DopriMix).
template <int D, int KIND, int MINB>
__global__ void __launch_bounds__(64, MINB)
dopri_mix_kernel(ProbArgs P, MediumArgs med, BeamArgs B, TrajArgs T, OdeArgs o, int tt_len) {
    constexpr int ND = MState<D>::ND;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int64_t bl = blockIdx.x * (int64_t)blockDim.x + threadIdx.x - stride;
    bool active = false;
    DopriMix<D, KIND> s;
    s.k64 = dopri_stage_smem + threadIdx.x;
    s.k32 = reinterpret_cast<float *>(dopri_stage_smem + 7 * ND * DopriMix<D, KIND>::kst) + threadIdx.x;
    RecordWriter<D> rw(P, T, 0, 0.0, tt_len);
    unsigned long long lane_steps = 0;
    for (;;) {
        if (!active) {
            bl += stride;
            while (bl < T.nb && o.only_flagged && T.status[bl] == 0) bl += stride;  // already accepted
            if (bl < T.nb) {
                double mode, w;
                State<D> y0;
                launch_state<D>(B, T, bl, y0, mode, w);
                mix_from_full(y0, s.y);
                rw.reset(bl, w);
                rw.put(0, y0, false);
                s.init(med, P, o, mode);
                active = true;
            }
        }
        if (!__any_sync(0xffffffffu, active)) break;
        if (active && s.attempt(med, P, o, rw)) {
            constexpr int S = MState<D>::S;
            bool fin = isfinite(s.y.f[2 * S]) && isfinite(s.y.f[2 * S + 1]);
#pragma unroll
            for (int c = 0; c < ND; ++c) fin = fin && isfinite(s.y.r[c]);
            if (!fin && s.code == 0) s.code = 1;
            if (s.k < P.nt) {  // after a failure: the last state
                State<D> yf;
                mix_to_full(s.y, yf);
                for (int64_t k = s.k; k < P.nt; ++k) rw.put(k, yf, true);
            }
            if (T.status) T.status[bl] = s.code;
            lane_steps += (unsigned long long)s.steps;
            active = false;
        }
    }
    if (o.step_count) {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) lane_steps += __shfl_xor_sync(0xffffffffu, lane_steps, off);
        if ((threadIdx.x & 31) == 0 && lane_steps) atomicAdd(o.step_count, lane_steps);
    }
}

// Fixed-step RK4, one thread per beam.
template <int D>
__global__ void rk4_kernel(ProbArgs P, MediumArgs med, BeamArgs B, TrajArgs T, OdeArgs o, int tt_len) {
    const int64_t bl = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (bl >= T.nb) return;
    if (o.only_flagged && T.status[bl] == 0) return;  // records already accepted
    const int64_t b = T.b_first + bl;
    const int64_t j = b < B.n ? b : b - B.n;
    const double mode = b < B.n ? 1.0 : -1.0;
    State<D> y;
#pragma unroll
    for (int i = 0; i < D; ++i) {
        y.x[i] = B.x0[j * D + i];
        y.p[i] = B.p0[j * D + i];
#pragma unroll
        for (int k = 0; k < D; ++k) y.M[i][k] = cd{0.0, 0.0};
        y.M[i][i] = cd{B.alpha[2 * (j * D + i)], B.alpha[2 * (j * D + i) + 1]};
    }
    y.A = cd{1.0, 0.0};
    const double w = B.omega[j];
    int code = 0;
    RecordWriter<D> rw(P, T, bl, w, tt_len);
    const int64_t n_tt = (P.nt + tt_len - 1) / tt_len;
    for (int64_t k = 0; k < P.nt; ++k) {
        if (k > 0 && code == 0) {
            const double hs = (P.ts[k] - P.ts[k - 1]) / o.substeps;
            for (int s = 0; s < o.substeps; ++s) rk4_step<D>(med, mode, y, hs);
        }
        bool fin = isfinite(y.A.re) && isfinite(y.A.im);
#pragma unroll
        for (int i = 0; i < D; ++i) fin = fin && isfinite(y.x[i]) && isfinite(y.p[i]);
        if (!fin && code == 0) code = 1;
        rw.put(k, y, code != 0);
    }
    (void)n_tt;
    if (T.status) T.status[bl] = code;
}

// Time reversal: beam i starts on the detector at t0[i] and runs back to
// t = 0.  With tau = t0 - t the state obeys dy/dtau = -f(y; mode, lam) =
// f(y; -mode, -lam) (every term of the right-hand side is odd in the branch
// except lam G / 2G), so the forward integrator runs unchanged over
// tau in [0, t0] on the flipped branch and absorption.
struct TrBeamsView {
    const double *x, *p, *M, *mode, *t0;
};

template <int D, int KIND>
__global__ void tr_final_kernel(ProbArgs P, MediumArgs med, TrBeamsView B, int64_t n, OdeArgs o, double *rec64,
                                int32_t *status) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    DopriBeam<D, KIND> s;
    s.ks = dopri_stage_smem + threadIdx.x;
    s.kst = blockDim.x;
#pragma unroll
    for (int a = 0; a < D; ++a) {
        s.y.x[a] = B.x[i * D + a];
        s.y.p[a] = B.p[i * D + a];
#pragma unroll
        for (int b = a; b < D; ++b)
            s.y.M[sym_index<D>(a, b)] = cd{B.M[2 * ((i * D + a) * D + b)], B.M[2 * ((i * D + a) * D + b) + 1]};
    }
    s.y.A = cd{1.0, 0.0};
    const double t0 = B.t0[i];
    int code = 0;
    if (t0 > 0.0) {
        double tl[2] = {0.0, t0};
        ProbArgs Pl = P;
        Pl.nt = 2;
        Pl.ts = tl;
        TrajArgs T{n, 0, n, nullptr, nullptr, nullptr, nullptr};  // records written below
        RecordWriter<D> rw(Pl, T, i, 1.0, 2);
        s.init(med, Pl, o, -B.mode[i]);
        while (!s.attempt(med, Pl, o, rw)) {
        }
        code = s.code;
    }
    bool fin = isfinite(s.y.A.re) && isfinite(s.y.A.im);
#pragma unroll
    for (int a = 0; a < D; ++a) fin = fin && isfinite(s.y.x[a]) && isfinite(s.y.p[a]);
    if (!fin && code == 0) code = 1;
    double *r = rec64 + i * (int64_t)NV<D>::value;
    State<D> yf;
    to_full(s.y, yf);
    const double *v = vals(yf);
#pragma unroll
    for (int c = 0; c < NV<D>::value; ++c) r[c] = v[c];
    status[i] = code;
}

// The integrator kernels specialised for the medium kind (run-time kind ->
// template argument).
struct Dopri {
    int minb;
    bool f32m;   // FP32 path: FP32 medium, and without dense output the mixed-precision state
    bool dense;  // save times from the continuous extension
    bool mixed() const { return f32m && !dense; }
    template <int D, int K>
    auto kernel() const {
        if (dense) return f32m ? dopri_kernel<D, K, 4, true, true> : dopri_kernel<D, K, 4, false, true>;
        if (f32m)
            return minb >= 7   ? dopri_mix_kernel<D, K, 7>
                   : minb == 6 ? dopri_mix_kernel<D, K, 6>
                   : minb == 5 ? dopri_mix_kernel<D, K, 5>
                               : dopri_mix_kernel<D, K, 4>;
        return minb >= 5 ? dopri_kernel<D, K, 5, false, false> : dopri_kernel<D, K, 4, false, false>;
    }
    template <int D>
    size_t smem() const { return mixed() ? dopri_mix_smem_bytes<D>(64) : dopri_smem_bytes<D>(64); }
};
struct TrFinal {
    template <int D, int K>
    auto kernel() const { return tr_final_kernel<D, K>; }
    template <int D>
    size_t smem() const { return dopri_smem_bytes<D>(64); }
};

// Blocks of 64 lanes per SM of the adaptive integrator: MSGB_DOPRI_BLOCKS
// (4 to 7; 5, 6 and 7 bound the registers to 204, 170 and 146; the FP64
// integrator takes at most 5), else `dflt`.
int dopri_blocks_per_sm(int dflt) {
    static const int env = [] {
        const char *e = getenv("MSGB_DOPRI_BLOCKS");
        const int v = e ? atoi(e) : 0;
        return (v >= 4 && v <= 7) ? v : 0;
    }();
    return env ? env : dflt;
}

template <int D, typename Launch, typename Which>
void launch_by_kind(int kind, Launch launch, const Which &which) {
    auto go = [&](auto kern) {
        const size_t smem = which.template smem<D>();
        if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        launch(kern, smem);
    };
    switch (kind) {
        case MSGB_MEDIUM_CONSTANT: go(which.template kernel<D, MSGB_MEDIUM_CONSTANT>()); break;
        case MSGB_MEDIUM_LINEAR: go(which.template kernel<D, MSGB_MEDIUM_LINEAR>()); break;
        default: go(which.template kernel<D, MSGB_MEDIUM_BSPLINE3>()); break;
    }
}

}  // namespace
}  // namespace msgb

using namespace msgb;

extern "C" int msgb_tr_final_states(const msgb_problem *prob, const msgb_medium *med, const msgb_tr_beams *beams,
                                    const msgb_ode_opts *opts, double *rec64, int32_t *status,
                                    msgb_stream_t stream) {
    if (!prob || !med || !beams || !opts) return fail(MSGB_ERR_ARG, "msgb_tr_final_states: NULL argument");
    if (prob->ndim < 1 || prob->ndim > 3) return fail(MSGB_ERR_ARG, "ndim must be 1, 2 or 3");
    if (beams->n < 0) return fail(MSGB_ERR_ARG, "negative beam count");
    if (opts->method != MSGB_ODE_DOPRI5) return fail(MSGB_ERR_ARG, "time reversal integrates with DOPRI5");
    if (!(opts->rtol > 0.0) || !(opts->atol > 0.0) || !isfinite(opts->rtol) || !isfinite(opts->atol))
        return fail(MSGB_ERR_ARG, "rtol and atol must be finite and positive");
    if (opts->max_steps < 1) return fail(MSGB_ERR_ARG, "max_steps must be a positive integer");
    if (!isfinite(opts->dt0)) return fail(MSGB_ERR_ARG, "dt0 must be finite");
    if (beams->n == 0) return MSGB_OK;
    if (!beams->x || !beams->p || !beams->M || !beams->mode || !beams->t0 || !rec64 || !status)
        return fail(MSGB_ERR_ARG, "msgb_tr_final_states: NULL array");
    MediumArgs M;
    if (int e = medium_args(prob, med, M)) return e;
    M.lam = -M.lam;
    ProbArgs P{};
    P.nd = prob->ndim;
    for (int a = 0; a < 3; ++a) {
        P.periodic[a] = a < prob->ndim ? (prob->periodic[a] != 0) : 0;
        P.L[a] = a < prob->ndim ? prob->L[a] : 1.0;
    }
    P.c = prob->c;
    OdeArgs O{opts->method, opts->substeps, opts->rtol, opts->atol, opts->dt0, opts->max_steps, 0,
              opts->dense_output, nullptr};
    TrBeamsView B{beams->x, beams->p, beams->M, beams->mode, beams->t0};
    const int blk = 64;
    const unsigned grid = (unsigned)((beams->n + blk - 1) / blk);
    cudaStream_t st = as_stream(stream);
    switch (prob->ndim) {
        case 1: launch_by_kind<1>(M.kind, [&](auto kern, size_t sm) { kern<<<grid, blk, sm, st>>>(P, M, B, beams->n, O, rec64, status); },
                                  TrFinal{}); break;
        case 2: launch_by_kind<2>(M.kind, [&](auto kern, size_t sm) { kern<<<grid, blk, sm, st>>>(P, M, B, beams->n, O, rec64, status); },
                                  TrFinal{}); break;
        default: launch_by_kind<3>(M.kind, [&](auto kern, size_t sm) { kern<<<grid, blk, sm, st>>>(P, M, B, beams->n, O, rec64, status); },
                                   TrFinal{}); break;
    }
    return check_launch("msgb_tr_final_states");
}

extern "C" int msgb_ode_trajectories(const msgb_problem *prob, const msgb_medium *med, const msgb_beam_set *beams,
                                     const msgb_ode_opts *opts, const msgb_trajectories *out,
                                     msgb_stream_t stream) {
    if (int e = validate_problem(prob)) return e;
    if (int e = validate_beams(prob, beams)) return e;
    if (!med || !out || !opts) return fail(MSGB_ERR_ARG, "msgb_ode_trajectories: NULL medium, options or output");
    if (opts->method == MSGB_ODE_RK4) {
        if (opts->substeps < 1) return fail(MSGB_ERR_ARG, "substeps must be >= 1");
    } else if (opts->method == MSGB_ODE_DOPRI5) {
        if (!(opts->rtol > 0.0) || !(opts->atol > 0.0) || !isfinite(opts->rtol) || !isfinite(opts->atol))
            return fail(MSGB_ERR_ARG, "rtol and atol must be finite and positive");
        if (opts->max_steps < 1) return fail(MSGB_ERR_ARG, "max_steps must be a positive integer");
        if (!isfinite(opts->dt0)) return fail(MSGB_ERR_ARG, "dt0 must be finite");
    } else {
        return fail(MSGB_ERR_ARG, "unknown ODE method %d", opts->method);
    }
    if (out->nb < 0 || out->b_first < 0 || out->b_first + out->nb > 2 * beams->n)
        return fail(MSGB_ERR_ARG, "beam range [%lld, %lld) outside [0, 2n)", (long long)out->b_first,
                    (long long)(out->b_first + out->nb));
    MediumArgs M;
    if (int e = medium_args(prob, med, M)) return e;
    if (out->nb == 0 || prob->nt == 0) return MSGB_OK;
    if (opts->only_flagged && !out->status)
        return fail(MSGB_ERR_ARG, "only_flagged needs the status array of the records");
    ProbArgs P = to_args(prob);
    OdeArgs O{opts->method, opts->substeps, opts->rtol, opts->atol, opts->dt0, opts->max_steps, opts->only_flagged,
              opts->dense_output, opts->step_count};
    if (int e = check_compact(out, prob->ndim)) return e;
    TrajArgs T{out->nb, out->b_first, beams->n, out->rec64, out->rec32, out->cull, out->status};
    set_compact(T, out);
    const int blk = 64;
    const int64_t need = (out->nb + blk - 1) / blk;
    cudaStream_t st = as_stream(stream);
    if (O.method == MSGB_ODE_RK4) {
        const unsigned grid = (unsigned)need;
        switch (prob->ndim) {
            case 1: rk4_kernel<1><<<grid, blk, 0, st>>>(P, M, to_args(beams), T, O, MSGB_TIME_TILE); break;
            case 2: rk4_kernel<2><<<grid, blk, 0, st>>>(P, M, to_args(beams), T, O, MSGB_TIME_TILE); break;
            default: rk4_kernel<3><<<grid, blk, 0, st>>>(P, M, to_args(beams), T, O, MSGB_TIME_TILE); break;
        }
    } else {
        // enough resident lanes for every SM, each taking several beams
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const bool f32m = opts->medium_fp32 != 0 && med->coeffs32 != nullptr && med->kind != MSGB_MEDIUM_CONSTANT;
        Dopri which{4, f32m, opts->dense_output != 0};
        which.minb = dopri_blocks_per_sm(which.mixed() ? kMixBlocks : 4);
        if (!which.mixed() && which.minb > 5) which.minb = 5;
        {
            // the lanes are persistent: every block must be resident at once
            const size_t sm_bytes = prob->ndim == 1 ? which.smem<1>() : (prob->ndim == 2 ? which.smem<2>() : which.smem<3>());
            const int fit = (int)((size_t)(227 * 1024) / sm_bytes);
            if (which.minb > fit) which.minb = fit < 4 ? 4 : fit;
        }
        const int64_t want = (int64_t)which.minb * sms;
        const unsigned grid = (unsigned)(need < want ? need : want);
        switch (prob->ndim) {
            case 1: launch_by_kind<1>(M.kind, [&](auto kern, size_t sm) { kern<<<grid, blk, sm, st>>>(P, M, to_args(beams), T, O, MSGB_TIME_TILE); },
                                      which); break;
            case 2: launch_by_kind<2>(M.kind, [&](auto kern, size_t sm) { kern<<<grid, blk, sm, st>>>(P, M, to_args(beams), T, O, MSGB_TIME_TILE); },
                                      which); break;
            default: launch_by_kind<3>(M.kind, [&](auto kern, size_t sm) { kern<<<grid, blk, sm, st>>>(P, M, to_args(beams), T, O, MSGB_TIME_TILE); },
                                       which); break;
        }
    }
    return check_launch("msgb_ode_trajectories");
}

extern "C" int msgb_rk4_trajectories(const msgb_problem *prob, const msgb_medium *med, const msgb_beam_set *beams,
                                     int substeps, const msgb_trajectories *out, msgb_stream_t stream) {
    msgb_ode_opts o{};
    o.method = MSGB_ODE_RK4;
    o.substeps = substeps;
    return msgb_ode_trajectories(prob, med, beams, &o, out, stream);
}
