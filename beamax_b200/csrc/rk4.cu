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
#include "common.cuh"

namespace msgb {
namespace {

struct MediumArgs {
    int kind, boundary;
    int n[3];
    double spacing[3], origin[3];
    const double *coeffs;
    double c, lam;
};

__device__ __forceinline__ int map_index(int i, int n, int boundary) {
    if (n == 1) return 0;
    switch (boundary) {
        case 0: return i < 0 ? 0 : (i > n - 1 ? n - 1 : i);
        case 1: { int r = i % n; return r < 0 ? r + n : r; }
        case 2: { const int per = 2 * n; int r = i % per; if (r < 0) r += per; return r < n ? r : per - 1 - r; }
        default: { const int per = 2 * n - 2; int r = i % per; if (r < 0) r += per; return r < n ? r : per - r; }
    }
}

// c, grad c (D), hess c (D x D, row-major) at x.
template <int D>
__device__ void speed_eval(const MediumArgs &m, const double *x, double &c, double *g, double *H) {
    if (m.kind == MSGB_MEDIUM_CONSTANT) {
        c = m.c;
#pragma unroll
        for (int i = 0; i < D; ++i) {
            g[i] = 0.0;
#pragma unroll
            for (int k = 0; k < D; ++k) H[i * D + k] = 0.0;
        }
        return;
    }
    const bool cubic = m.kind == MSGB_MEDIUM_BSPLINE3;
    const int taps = cubic ? 4 : 2;
    const int off0 = cubic ? -1 : 0;
    double w[D][4], d1[D][4], d2[D][4];
    int idx[D][4];
#pragma unroll
    for (int a = 0; a < D; ++a) {
        const double u = (x[a] - m.origin[a]) / m.spacing[a];
        const double fl = floor(u);
        const double t = u - fl;
        const int i0 = (int)fl;
        if (cubic) {
            const double omt = 1.0 - t, t2 = t * t, t3 = t2 * t;
            w[a][0] = omt * omt * omt / 6.0;
            w[a][1] = (3.0 * t3 - 6.0 * t2 + 4.0) / 6.0;
            w[a][2] = (-3.0 * t3 + 3.0 * t2 + 3.0 * t + 1.0) / 6.0;
            w[a][3] = t3 / 6.0;
            d1[a][0] = -(omt * omt) / 2.0;
            d1[a][1] = 1.5 * t2 - 2.0 * t;
            d1[a][2] = -1.5 * t2 + t + 0.5;
            d1[a][3] = t2 / 2.0;
            d2[a][0] = omt;
            d2[a][1] = 3.0 * t - 2.0;
            d2[a][2] = -3.0 * t + 1.0;
            d2[a][3] = t;
        } else {
            w[a][0] = 1.0 - t;
            w[a][1] = t;
            d1[a][0] = -1.0;
            d1[a][1] = 1.0;
            d2[a][0] = d2[a][1] = 0.0;
            w[a][2] = w[a][3] = d1[a][2] = d1[a][3] = d2[a][2] = d2[a][3] = 0.0;
        }
        for (int k = 0; k < taps; ++k) idx[a][k] = map_index(i0 + off0 + k, m.n[a], m.boundary);
    }
    double cc = 0.0, gg[D], hh[D][D];
#pragma unroll
    for (int i = 0; i < D; ++i) {
        gg[i] = 0.0;
#pragma unroll
        for (int k = 0; k < D; ++k) hh[i][k] = 0.0;
    }
    const int ncorner = D == 1 ? taps : (D == 2 ? taps * taps : taps * taps * taps);
    for (int corner = 0; corner < ncorner; ++corner) {
        int loc[D];
        int rem = corner;
        int64_t flat = 0;
#pragma unroll
        for (int a = D - 1; a >= 0; --a) {
            loc[a] = rem % taps;
            rem /= taps;
        }
#pragma unroll
        for (int a = 0; a < D; ++a) flat = flat * m.n[a] + idx[a][loc[a]];
        const double v = __ldg(m.coeffs + flat);
        double wall = 1.0;
#pragma unroll
        for (int a = 0; a < D; ++a) wall *= w[a][loc[a]];
        cc = fma(wall, v, cc);
#pragma unroll
        for (int a = 0; a < D; ++a) {
            double ga = d1[a][loc[a]];
            double ha = d2[a][loc[a]];
#pragma unroll
            for (int o = 0; o < D; ++o)
                if (o != a) {
                    ga *= w[o][loc[o]];
                    ha *= w[o][loc[o]];
                }
            gg[a] = fma(ga, v, gg[a]);
            hh[a][a] = fma(ha, v, hh[a][a]);
#pragma unroll
            for (int b = a + 1; b < D; ++b) {
                double hab = d1[a][loc[a]] * d1[b][loc[b]];
#pragma unroll
                for (int o = 0; o < D; ++o)
                    if (o != a && o != b) hab *= w[o][loc[o]];
                hh[a][b] = fma(hab, v, hh[a][b]);
            }
        }
    }
    c = cc;
#pragma unroll
    for (int a = 0; a < D; ++a) {
        g[a] = gg[a] / m.spacing[a];
#pragma unroll
        for (int b = 0; b < D; ++b) {
            const double hv = a <= b ? hh[a][b] : hh[b][a];
            H[a * D + b] = hv / (m.spacing[a] * m.spacing[b]);
        }
    }
}

template <int D>
struct State {
    double x[D], p[D];
    cd M[D][D];
    cd A;
};

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
};

template <int D>
struct NV {
    static constexpr int value = 2 * D + 2 * D * D + 2;  // doubles in State<D>
};

template <int D>
__device__ __forceinline__ double *vals(State<D> &s) { return reinterpret_cast<double *>(&s); }
template <int D>
__device__ __forceinline__ const double *vals(const State<D> &s) { return reinterpret_cast<const double *>(&s); }

// Magnitude of complex entry e of the state (x and p entries are real).
template <int D>
__device__ __forceinline__ double entry_abs(const double *v, int e) {
    if (e < 2 * D) return fabs(v[e]);
    const int q = 2 * D + 2 * (e - 2 * D);
    return hypot(v[q], v[q + 1]);
}

// One adaptive step attempt sequence from t to t_end.  Returns 0, or 2 when
// the step budget runs out (the state then stays at the last accepted step).
template <int D>
__device__ int dopri_advance(const MediumArgs &med, double mode, State<D> &y, State<D> &f0, double &t,
                             const double t_end, double &h, int64_t &steps, const OdeArgs &o) {
    constexpr int N = NV<D>::value;
    constexpr int NE = 2 * D + D * D + 1;
    static_assert(sizeof(State<D>) == N * sizeof(double), "State<D> must be a plain array of doubles");
    while (t < t_end) {
        if (steps >= o.max_steps) return 2;
        double hh = h;
        bool clipped = false;
        if (t + hh >= t_end) {
            hh = t_end - t;
            clipped = true;
        }
        State<D> k[7];
        k[0] = f0;
        State<D> yt;
        const double *yv = vals(y);
#pragma unroll 1
        for (int s = 1; s < 7; ++s) {
            double *tv = vals(yt);
#pragma unroll
            for (int c = 0; c < N; ++c) {
                double acc = 0.0;
                for (int j = 0; j < s; ++j) {
                    const double a = DP_A[s][j];
                    if (a != 0.0) acc += a * vals(k[j])[c];
                }
                tv[c] = yv[c] + hh * acc;
            }
            rhs<D>(med, mode, yt, k[s]);
        }
        // yt now holds the 5th-order solution (stage 7's input).
        double ev[N];
#pragma unroll
        for (int c = 0; c < N; ++c) {
            double acc = 0.0;
            for (int j = 0; j < 7; ++j) acc += DP_E[j] * vals(k[j])[c];
            ev[c] = hh * acc;
        }
        double sum = 0.0;
        const double *nv = vals(yt);
#pragma unroll
        for (int e = 0; e < NE; ++e) {
            const double sc = o.atol + o.rtol * fmax(entry_abs<D>(yv, e), entry_abs<D>(nv, e));
            const double r = entry_abs<D>(ev, e) / sc;
            sum += r * r;
        }
        const double err = sqrt(sum / NE);
        ++steps;
        if (!isfinite(err)) {
            h = 0.2 * hh;
            continue;
        }
        const double fac = err == 0.0 ? 10.0 : fmin(10.0, fmax(0.2, 0.9 * pow(err, -0.2)));
        if (err <= 1.0) {
            t = clipped ? t_end : t + hh;
            y = yt;
            f0 = k[6];
            const double hn = hh * fac;
            h = clipped ? fmax(hn, h) : hn;
        } else {
            h = hh * fmin(1.0, fac);
        }
    }
    return 0;
}

// Smallest eigenvalue of a symmetric D x D matrix (exact for D <= 2,
// Gershgorin lower bound for D = 3).
template <int D>
__device__ __forceinline__ double lam_min(const double (*S)[D]) {
    if (D == 1) return S[0][0];
    if (D == 2) {
        const double a = S[0][0], b = 0.5 * (S[0][1 % D] + S[1 % D][0]), c = S[1 % D][1 % D];
        const double m = 0.5 * (a + c), r = sqrt(0.25 * (a - c) * (a - c) + b * b);
        return m - r;
    }
    double lo = 1e300;
#pragma unroll
    for (int i = 0; i < D; ++i) {
        double s = S[i][i];
#pragma unroll
        for (int k = 0; k < D; ++k)
            if (k != i) s -= fabs(0.5 * (S[i][k] + S[k][i]));
        lo = fmin(lo, s);
    }
    return lo;
}

struct TrajArgs {
    int64_t nb, b_first, n;
    double *rec64;
    void *rec32;
    float *cull;
    int32_t *status;
};

template <int D>
__global__ void ode_kernel(ProbArgs P, MediumArgs med, BeamArgs B, TrajArgs T, OdeArgs o, int tt_len) {
    const int64_t bl = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (bl >= T.nb) return;
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
    const bool adaptive = o.method == MSGB_ODE_DOPRI5;
    double h = o.dt0 > 0.0 ? o.dt0 : (P.nt > 1 ? P.ts[1] - P.ts[0] : 0.0);
    double t = P.ts[0];
    int64_t steps = 0;
    int code = 0;
    State<D> f0;
    if (adaptive) rhs<D>(med, mode, y, f0);
    constexpr int S = D * (D + 1) / 2;
    constexpr int NR64 = 2 * D + 2 * D * D + 2;
    float lo[D], hi[D];
    double lmin = 1e300;
    bool bad = false;
    const int64_t n_tt = (P.nt + tt_len - 1) / tt_len;
    for (int64_t k = 0; k < P.nt; ++k) {
        if (k > 0 && code == 0) {
            if (adaptive) {
                code = dopri_advance<D>(med, mode, y, f0, t, P.ts[k], h, steps, o);
            } else {
                const double hs = (P.ts[k] - P.ts[k - 1]) / o.substeps;
                for (int s = 0; s < o.substeps; ++s) rk4_step<D>(med, mode, y, hs);
            }
        }
        bool fin = isfinite(y.A.re) && isfinite(y.A.im);
#pragma unroll
        for (int i = 0; i < D; ++i) fin = fin && isfinite(y.x[i]) && isfinite(y.p[i]);
        if (!fin && code == 0) code = 1;
        bad |= code != 0;
        double xw[D];
#pragma unroll
        for (int i = 0; i < D; ++i) xw[i] = P.periodic[i] ? pymod(y.x[i], P.L[i]) : y.x[i];
        if (T.rec64) {
            double *r = T.rec64 + (k * T.nb + bl) * NR64;
            int q = 0;
#pragma unroll
            for (int i = 0; i < D; ++i) r[q++] = y.x[i];
#pragma unroll
            for (int i = 0; i < D; ++i) r[q++] = y.p[i];
#pragma unroll
            for (int i = 0; i < D; ++i)
#pragma unroll
                for (int l = 0; l < D; ++l) {
                    r[q++] = y.M[i][l].re;
                    r[q++] = y.M[i][l].im;
                }
            r[q++] = y.A.re;
            r[q++] = y.A.im;
        }
        if (T.rec32) {
            // layout of the FP32 summation's BeamTime<D> record
            char *base = (char *)T.rec32 + (k * T.nb + bl) * (int64_t)(16 * D + 8 * S + 8);
            double *xd = (double *)base;
            double *wpd = xd + D;
            float *f = (float *)(wpd + D);
#pragma unroll
            for (int i = 0; i < D; ++i) {
                xd[i] = xw[i];
                wpd[i] = w * y.p[i];
            }
#pragma unroll
            for (int i = 0; i < D; ++i)
#pragma unroll
                for (int l = i; l < D; ++l) {
                    const int q = sym_index<D>(i, l);
                    const double fac = (i == l ? 0.5 : 0.5) * w;  // off-diagonal: (M_il + M_li)/2 doubled
                    const double mre = i == l ? y.M[i][i].re : (y.M[i][l].re + y.M[l][i].re);
                    const double mim = i == l ? y.M[i][i].im : (y.M[i][l].im + y.M[l][i].im);
                    f[q] = (float)(fac * mre);
                    f[S + q] = (float)(fac * mim);
                }
            f[2 * S] = (float)atan2(y.A.im, (y.A.re == 0.0 && y.A.im == 0.0) ? 1e-12 : y.A.re);
            f[2 * S + 1] = (float)(2.0 * hypot(y.A.re, y.A.im));
        }
        if (T.cull) {
            double Sm[D][D];
#pragma unroll
            for (int i = 0; i < D; ++i)
#pragma unroll
                for (int l = 0; l < D; ++l) Sm[i][l] = y.M[i][l].im;
            const int kk = (int)(k % tt_len);
            if (kk == 0) {
                lmin = 1e300;
#pragma unroll
                for (int i = 0; i < D; ++i) lo[i] = 3.4e38f, hi[i] = -3.4e38f;
            }
            lmin = fmin(lmin, lam_min<D>(Sm));
#pragma unroll
            for (int i = 0; i < D; ++i) {
                const float xf = (float)xw[i];
                lo[i] = fminf(lo[i], xf);
                hi[i] = fmaxf(hi[i], xf);
            }
            if (kk == tt_len - 1 || k == P.nt - 1) {
                float *c = T.cull + ((k / tt_len) * T.nb + bl) * (2 * D + 1);
#pragma unroll
                for (int i = 0; i < D; ++i) {
                    // periodic axes and non-finite states are never culled
                    const bool open = P.periodic[i] || bad;
                    c[i] = open ? -3.4e38f : lo[i];
                    c[D + i] = open ? 3.4e38f : hi[i];
                }
                c[2 * D] = bad ? 0.0f : (float)fmax(0.0, 0.5 * w * lmin * (1.0 - 1e-6));
            }
        }
    }
    (void)n_tt;
    if (T.status) T.status[bl] = code;
}

}  // namespace
}  // namespace msgb

using namespace msgb;

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
    if (med->kind != MSGB_MEDIUM_CONSTANT) {
        if (med->kind != MSGB_MEDIUM_LINEAR && med->kind != MSGB_MEDIUM_BSPLINE3)
            return fail(MSGB_ERR_ARG, "unknown medium kind %d", med->kind);
        if (!med->coeffs) return fail(MSGB_ERR_ARG, "medium grid is NULL");
        if (med->boundary < 0 || med->boundary > 3) return fail(MSGB_ERR_ARG, "unknown boundary %d", med->boundary);
        for (int a = 0; a < prob->ndim; ++a)
            if (med->n[a] < 1 || !(med->spacing[a] > 0.0)) return fail(MSGB_ERR_ARG, "bad medium grid");
    } else if (!(med->c > 0.0)) {
        return fail(MSGB_ERR_ARG, "constant medium speed must be > 0");
    }
    if (out->nb == 0 || prob->nt == 0) return MSGB_OK;
    ProbArgs P = to_args(prob);
    MediumArgs M{};
    M.kind = med->kind;
    M.boundary = med->boundary;
    for (int a = 0; a < 3; ++a) {
        M.n[a] = med->n[a];
        M.spacing[a] = med->spacing[a];
        M.origin[a] = med->origin[a];
    }
    M.coeffs = med->coeffs;
    M.c = med->c;
    M.lam = med->lam;
    OdeArgs O{opts->method, opts->substeps, opts->rtol, opts->atol, opts->dt0, opts->max_steps};
    TrajArgs T{out->nb, out->b_first, beams->n, out->rec64, out->rec32, out->cull, out->status};
    const int blk = 64;
    const unsigned grid = (unsigned)((out->nb + blk - 1) / blk);
    cudaStream_t st = as_stream(stream);
    switch (prob->ndim) {
        case 1: ode_kernel<1><<<grid, blk, 0, st>>>(P, M, to_args(beams), T, O, MSGB_TIME_TILE); break;
        case 2: ode_kernel<2><<<grid, blk, 0, st>>>(P, M, to_args(beams), T, O, MSGB_TIME_TILE); break;
        default: ode_kernel<3><<<grid, blk, 0, st>>>(P, M, to_args(beams), T, O, MSGB_TIME_TILE); break;
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
