/*
 * FP64 C/OpenMP restatement of the heterogeneous MSGB beam path (test oracle
 * and timed CPU baseline; never linked into the product).
 *
 * Restates:
 *   utils/interp.py:31-263     make_c_function_from_grid: n-linear or cubic
 *                              B-spline tensor product on prefiltered
 *                              coefficients, boundary maps :78-98, weights
 *                              :101-118; gradient and Hessian are the exact
 *                              derivatives of that formula (jax.grad/hessian).
 *   gb/gb_solvers.py:787-867   riccati_rhs + coupled_rhs_absorption.
 *   gb/gb_solvers.py:597-784,940-1014  solve_ODE_base: adaptive integration
 *                              with SaveAt(ts).  The reference runs diffrax
 *                              Tsit5 with PIDController(rtol, atol) (diffrax
 *                              0.7.2, not installed here); this restates the
 *                              same control (RMS error norm over the complex
 *                              state, factor clip(0.9 err^-1/5, 0.2, 10), no
 *                              growth right after a rejection, dt0 = ts[1] -
 *                              ts[0], the max_steps budget) on the
 *                              Dormand-Prince 5(4) pair, step for step as
 *                              oracle/ode.py:dopri5 does; steps end on the
 *                              save times.
 *   gb/core.py:194-329         compute_gaussian_beam_real on the trajectories
 *                              (dense: every beam, time and sensor).
 * and the exact transpose of that sum down to each beam's amplitude:
 *   g_b = sum_{t,s} 2 d(t,s) conj(K_b(t,s)),  contribution = 2 Re[a_b K_b].
 *
 * State layout (per beam and save time), the rec64 layout of the CUDA
 * integrator: x (d), p (d), M (d x d row-major, re/im interleaved), A (re, im);
 * 2d + 2d^2 + 2 doubles.  The amplitude is integrated from a_init.
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

typedef double complex cplx;

typedef struct {
    int kind;          /* 0 constant, 1 linear, 2 cubic B-spline */
    int boundary;      /* 0 nearest, 1 wrap, 2 reflect, 3 mirror */
    int n[3];
    double spacing[3], origin[3];
    const double *coeffs;
    double c, lam;
} oracle_medium;

static int map_index(int i, int n, int boundary) {
    if (n == 1) return 0;
    switch (boundary) {
        case 0: return i < 0 ? 0 : (i > n - 1 ? n - 1 : i);
        case 1: { int r = i % n; return r < 0 ? r + n : r; }
        case 2: { int per = 2 * n, r = i % per; if (r < 0) r += per; return r < n ? r : per - 1 - r; }
        default: { int per = 2 * n - 2, r = i % per; if (r < 0) r += per; return r < n ? r : per - r; }
    }
}

/* c, grad c, Hessian c at x (interp.py:121-155 tensor product, summed over
 * every corner of the stencil). */
static void speed(int d, const oracle_medium *m, const double *x, double *c, double *g, double *H) {
    for (int a = 0; a < d; ++a) {
        g[a] = 0.0;
        for (int b = 0; b < d; ++b) H[a * d + b] = 0.0;
    }
    if (m->kind == 0) {
        *c = m->c;
        return;
    }
    const int cubic = m->kind == 2;
    const int taps = cubic ? 4 : 2, off0 = cubic ? -1 : 0;
    double w[3][4], d1[3][4], d2[3][4];
    int idx[3][4];
    for (int a = 0; a < d; ++a) {
        double u = (x[a] - m->origin[a]) / m->spacing[a];
        double fl = floor(u), t = u - fl;
        int i0 = (int)fl;
        if (cubic) {
            double omt = 1.0 - t, t2 = t * t, t3 = t2 * t;
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
        }
        for (int k = 0; k < taps; ++k) idx[a][k] = map_index(i0 + off0 + k, m->n[a], m->boundary);
    }
    double cc = 0.0;
    int corners = 1;
    for (int a = 0; a < d; ++a) corners *= taps;
    for (int corner = 0; corner < corners; ++corner) {
        int loc[3], rem = corner;
        int64_t flat = 0;
        for (int a = d - 1; a >= 0; --a) {
            loc[a] = rem % taps;
            rem /= taps;
        }
        for (int a = 0; a < d; ++a) flat = flat * m->n[a] + idx[a][loc[a]];
        double v = m->coeffs[flat];
        double wp = 1.0;
        for (int a = 0; a < d; ++a) wp *= w[a][loc[a]];
        cc += wp * v;
        for (int a = 0; a < d; ++a) {
            double ga = d1[a][loc[a]];
            for (int e = 0; e < d; ++e)
                if (e != a) ga *= w[e][loc[e]];
            g[a] += ga * v / m->spacing[a];
            for (int b = 0; b < d; ++b) {
                double hab;
                if (a == b) {
                    hab = d2[a][loc[a]];
                    for (int e = 0; e < d; ++e)
                        if (e != a) hab *= w[e][loc[e]];
                } else {
                    hab = d1[a][loc[a]] * d1[b][loc[b]];
                    for (int e = 0; e < d; ++e)
                        if (e != a && e != b) hab *= w[e][loc[e]];
                }
                H[a * d + b] += hab * v / (m->spacing[a] * m->spacing[b]);
            }
        }
    }
    *c = cc;
}

/* Packed real state: x (d), p (d), Re M (d^2), Im M (d^2), Re A, Im A. */
#define NV(d) (2 * (d) + 2 * (d) * (d) + 2)

/* coupled_rhs_absorption (gb_solvers.py:820-867) with riccati_rhs (:787-817). */
static void rhs(int d, const oracle_medium *m, double mode, const double *y, double *dy) {
    const double *x = y, *p = y + d;
    cplx M[3][3], A = y[NV(d) - 2] + I * y[NV(d) - 1];
    for (int i = 0; i < d; ++i)
        for (int k = 0; k < d; ++k) M[i][k] = y[2 * d + i * d + k] + I * y[2 * d + d * d + i * d + k];
    double c, gc[3], hc[9];
    speed(d, m, x, &c, gc, hc);
    double n2 = 0.0;
    for (int i = 0; i < d; ++i) n2 += p[i] * p[i];
    double np_ = sqrt(n2), np3 = np_ * n2;
    double G = mode * c * np_, Gx[3], Gp[3], Gpp[3][3], Gxp[3][3], Gxx[3][3];
    for (int i = 0; i < d; ++i) {
        Gx[i] = mode * gc[i] * np_;
        Gp[i] = mode * c * p[i] / np_;
    }
    for (int i = 0; i < d; ++i)
        for (int k = 0; k < d; ++k) {
            Gpp[i][k] = mode * c * ((i == k ? 1.0 : 0.0) / np_ - p[i] * p[k] / np3);
            Gxp[i][k] = mode * gc[i] * p[k] / np_;
            Gxx[i][k] = mode * hc[i * d + k] * np_;
        }
    cplx MG[3][3];
    for (int i = 0; i < d; ++i)
        for (int k = 0; k < d; ++k) {
            cplx s = 0.0;
            for (int l = 0; l < d; ++l) s += M[i][l] * Gpp[l][k];
            MG[i][k] = s;
        }
    for (int i = 0; i < d; ++i)
        for (int k = 0; k < d; ++k) {
            cplx s = Gxx[i][k];
            for (int l = 0; l < d; ++l) s += Gxp[i][l] * M[l][k] + M[i][l] * Gxp[k][l] + MG[i][l] * M[l][k];
            dy[2 * d + i * d + k] = -creal(s);
            dy[2 * d + d * d + i * d + k] = -cimag(s);
        }
    cplx trM = 0.0, gpmgp = 0.0;
    double gxgp = 0.0;
    for (int i = 0; i < d; ++i) {
        trM += M[i][i];
        gxgp += Gx[i] * Gp[i];
        for (int k = 0; k < d; ++k) gpmgp += Gp[i] * M[i][k] * Gp[k];
    }
    cplx dA = -A * (c * c * trM - gxgp - gpmgp + m->lam * G) / (2.0 * G);
    for (int i = 0; i < d; ++i) {
        dy[i] = Gp[i];
        dy[d + i] = -Gx[i];
    }
    dy[NV(d) - 2] = creal(dA);
    dy[NV(d) - 1] = cimag(dA);
}

/* Dormand & Prince (1980) 5(4): stage matrix, 5th-order weights, error
 * weights (5th minus 4th order). */
static const double DPA[7][6] = {
    {0, 0, 0, 0, 0, 0},
    {1.0 / 5, 0, 0, 0, 0, 0},
    {3.0 / 40, 9.0 / 40, 0, 0, 0, 0},
    {44.0 / 45, -56.0 / 15, 32.0 / 9, 0, 0, 0},
    {19372.0 / 6561, -25360.0 / 2187, 64448.0 / 6561, -212.0 / 729, 0, 0},
    {9017.0 / 3168, -355.0 / 33, 46732.0 / 5247, 49.0 / 176, -5103.0 / 18656, 0},
    {35.0 / 384, 0, 500.0 / 1113, 125.0 / 192, -2187.0 / 6784, 11.0 / 84}};
static const double DPB[7] = {35.0 / 384, 0, 500.0 / 1113, 125.0 / 192, -2187.0 / 6784, 11.0 / 84, 0};
static const double DPBH[7] = {5179.0 / 57600, 0, 7571.0 / 16695, 393.0 / 640, -92097.0 / 339200,
                               187.0 / 2100, 1.0 / 40};

/* RMS over the complex entries (x, p real; M, A complex) of |e| / (atol +
 * rtol max(|y0|, |y1|)): optimistix.rms_norm as diffrax's PIDController uses it. */
static double error_norm(int d, const double *e, const double *y0, const double *y1, double rtol, double atol) {
    double sum = 0.0;
    int cnt = 0;
    for (int i = 0; i < 2 * d; ++i, ++cnt) {
        double r = fabs(e[i]) / (atol + rtol * fmax(fabs(y0[i]), fabs(y1[i])));
        sum += r * r;
    }
    for (int q = 0; q <= d * d; ++q, ++cnt) {
        int re = q < d * d ? 2 * d + q : NV(d) - 2;
        int im = q < d * d ? 2 * d + d * d + q : NV(d) - 1;
        double r = hypot(e[re], e[im]) / (atol + rtol * fmax(hypot(y0[re], y0[im]), hypot(y1[re], y1[im])));
        sum += r * r;
    }
    return sqrt(sum / cnt);
}

static void put_record(int d, const double *y, double *rec) {
    int q = 0;
    for (int i = 0; i < 2 * d; ++i) rec[q++] = y[i];
    for (int i = 0; i < d * d; ++i) {
        rec[q++] = y[2 * d + i];
        rec[q++] = y[2 * d + d * d + i];
    }
    rec[q++] = y[NV(d) - 2];
    rec[q++] = y[NV(d) - 1];
}

/* One beam: states at every ts into rec (nt records).  Returns 0 ok, 1 non-finite
 * state, 2 step budget exhausted (later records hold the last state).
 * *steps_out: attempted steps. */
static int dopri5_beam(int d, const oracle_medium *m, double mode, const double *x0, const double *p0,
                       const cplx *m0diag, cplx a_init, int64_t nt, const double *ts, double rtol,
                       double atol, int64_t max_steps, double dt0, double *rec, int64_t *steps_out) {
    const int N = NV(d);
    double y[NV(3)], k[7][NV(3)], yt[NV(3)], y5[NV(3)], e[NV(3)];
    memset(y, 0, sizeof(y));
    for (int i = 0; i < d; ++i) {
        y[i] = x0[i];
        y[d + i] = p0[i];
        y[2 * d + i * d + i] = creal(m0diag[i]);
        y[2 * d + d * d + i * d + i] = cimag(m0diag[i]);
    }
    y[N - 2] = creal(a_init);
    y[N - 1] = cimag(a_init);
    const int RL = 2 * d + 2 * d * d + 2;
    put_record(d, y, rec);
    double h = dt0 > 0.0 ? dt0 : (nt > 1 ? ts[1] - ts[0] : 0.0);
    double t = ts[0];
    int64_t kk = 1, steps = 0, budget = max_steps + nt - 1;
    int rejected = 0, status = 0;
    rhs(d, m, mode, y, k[0]);
    while (kk < nt && status == 0) {
        if (steps >= budget) {
            status = 2;
            break;
        }
        double target = ts[kk], hh = h;
        int last = 0;
        if (t + hh >= target) {
            hh = target - t;
            last = 1;
        }
        for (int s = 1; s < 7; ++s) {
            for (int c = 0; c < N; ++c) {
                double acc = 0.0;
                for (int j = 0; j < s; ++j)
                    if (DPA[s][j] != 0.0) acc += DPA[s][j] * k[j][c];
                yt[c] = y[c] + hh * acc;
            }
            rhs(d, m, mode, yt, k[s]);
        }
        for (int c = 0; c < N; ++c) {
            double acc5 = 0.0, acce = 0.0;
            for (int j = 0; j < 7; ++j) {
                if (DPB[j] != 0.0) acc5 += DPB[j] * k[j][c];
                acce += (DPB[j] - DPBH[j]) * k[j][c];
            }
            y5[c] = y[c] + hh * acc5;
            e[c] = hh * acce;
        }
        double err = error_norm(d, e, y, y5, rtol, atol);
        ++steps;
        if (!isfinite(err)) {
            h = 0.2 * hh;
            rejected = 1;
            continue;
        }
        double fac = err == 0.0 ? 10.0 : fmin(10.0, fmax(0.2, 0.9 * pow(err, -0.2)));
        if (err <= 1.0) {
            if (rejected) fac = fmin(fac, 1.0);
            rejected = 0;
            double t_new = last ? target : t + hh;
            while (kk < nt && ts[kk] <= t_new) {
                put_record(d, y5, rec + kk * RL);  /* steps end on the save times */
                ++kk;
            }
            t = t_new;
            memcpy(y, y5, sizeof(double) * N);
            memcpy(k[0], k[6], sizeof(double) * N);
            h = last ? fmax(hh * fac, h) : hh * fac;
            for (int c = 0; c < N; ++c)
                if (!isfinite(y[c])) status = 1;
        } else {
            h = hh * fmin(1.0, fac);
            rejected = 1;
        }
    }
    for (; kk < nt; ++kk) put_record(d, y, rec + kk * RL);
    if (steps_out) *steps_out = steps;
    return status;
}

/* Trajectories of nb beams: beam i starts at x0[i], p0[i], M0 = diag(alpha[i])
 * (complex interleaved), A = 1, on branch mode[i].  rec: (nb, nt, 2d + 2d^2 + 2);
 * status: (nb).  steps: (nb) attempted steps (may be NULL). */
int oracle_het_traj(int d, int64_t nb, const double *x0, const double *p0, const double *alpha,
                    const double *mode, int kind, int boundary, const int *n, const double *spacing,
                    const double *origin, const double *coeffs, double c, double lam, double rtol, double atol,
                    int64_t max_steps, double dt0, int64_t nt, const double *ts, double *rec, int *status,
                    int64_t *steps) {
    if (d < 1 || d > 3) return 1;
    oracle_medium m;
    m.kind = kind;
    m.boundary = boundary;
    for (int a = 0; a < 3; ++a) {
        m.n[a] = n[a];
        m.spacing[a] = spacing[a];
        m.origin[a] = origin[a];
    }
    m.coeffs = coeffs;
    m.c = c;
    m.lam = lam;
    const int64_t RL = 2 * d + 2 * d * d + 2;
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t b = 0; b < nb; ++b) {
        cplx al[3];
        for (int i = 0; i < d; ++i) al[i] = alpha[2 * (b * d + i)] + I * alpha[2 * (b * d + i) + 1];
        int64_t st = 0;
        status[b] = dopri5_beam(d, &m, mode[b], x0 + b * d, p0 + b * d, al, 1.0, nt, ts, rtol, atol, max_steps,
                                dt0, rec + b * nt * RL, &st);
        if (steps) steps[b] = st;
    }
    return 0;
}

static double pymod(double a, double b) {
    double r = fmod(a, b);
    if (r != 0.0 && ((r < 0.0) != (b < 0.0))) r += b;
    return r;
}

/* Phase w (p.D + D^T Re M D / 2) + arg A and exponent w D^T Im M D / 2 of one
 * record at one sensor (gb/core.py:267-303, wrap_position :16-36). */
static void rec_terms(int d, const double *r, double w, const double *s, const double *L, const int *per,
                      double *phi, double *chi) {
    double D[3];
    for (int i = 0; i < d; ++i) {
        double xi = per[i] ? pymod(r[i], L[i]) : r[i];
        double di = s[i] - xi;
        if (per[i]) di = di - L[i] * nearbyint(di / L[i]);
        D[i] = di;
    }
    double lin = 0.0, qr = 0.0, qi = 0.0;
    for (int i = 0; i < d; ++i) lin += D[i] * r[d + i];
    for (int i = 0; i < d; ++i)
        for (int j = 0; j < d; ++j) {
            qr += D[i] * r[2 * d + 2 * (i * d + j)] * D[j];
            qi += D[i] * r[2 * d + 2 * (i * d + j) + 1] * D[j];
        }
    *phi = w * (lin + 0.5 * qr);
    *chi = w * 0.5 * qi;
}

/* Dense forward: out[t, s] += sum_b 2 |a_b A_b| cos(phi + arg(a_b A_b)) exp(-chi).
 * rec: (nb, nt, RL); amp: (nb) complex interleaved; omega: (nb). */
int oracle_sum_traj(int d, int64_t nb, const double *rec, const double *amp, const double *omega, int64_t nt,
                    int64_t ns, const double *sens, const double *L, const int *per, double *out) {
    if (d < 1 || d > 3) return 1;
    const int64_t RL = 2 * d + 2 * d * d + 2;
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t t = 0; t < nt; ++t) {
        double *row = out + t * ns;
        for (int64_t b = 0; b < nb; ++b) {
            const double *r = rec + (b * nt + t) * RL;
            cplx A = (amp[2 * b] + I * amp[2 * b + 1]) * (r[RL - 2] + I * r[RL - 1]);
            double re = creal(A), im = cimag(A);
            double ang = atan2(im, (re == 0.0 && im == 0.0) ? 1e-12 : re), mag = 2.0 * cabs(A);
            for (int64_t s = 0; s < ns; ++s) {
                double phi, chi;
                rec_terms(d, r, omega[b], sens + s * d, L, per, &phi, &chi);
                row[s] += mag * cos(phi + ang) * exp(-chi);
            }
        }
    }
    return 0;
}

/* Exact transpose: g[b] = sum_{t,s} 2 d(t,s) conj(A_b(t) e^{i phi - chi}) (the
 * derivative of the forward with respect to a_b, as a complex gradient). */
int oracle_adj_traj(int d, int64_t nb, const double *rec, const double *omega, int64_t nt, int64_t ns,
                    const double *sens, const double *L, const int *per, const double *data, double *g) {
    if (d < 1 || d > 3) return 1;
    const int64_t RL = 2 * d + 2 * d * d + 2;
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t b = 0; b < nb; ++b) {
        cplx acc = 0.0;
        for (int64_t t = 0; t < nt; ++t) {
            const double *r = rec + (b * nt + t) * RL;
            cplx ca = conj(r[RL - 2] + I * r[RL - 1]);
            const double *drow = data + t * ns;
            for (int64_t s = 0; s < ns; ++s) {
                double phi, chi;
                rec_terms(d, r, omega[b], sens + s * d, L, per, &phi, &chi);
                acc += 2.0 * drow[s] * ca * (cos(phi) - I * sin(phi)) * exp(-chi);
            }
        }
        g[2 * b] = creal(acc);
        g[2 * b + 1] = cimag(acc);
    }
    return 0;
}
