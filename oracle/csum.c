/*
 * FP64 C/OpenMP restatement of the reference's dense Gaussian-beam summation
 * (test oracle and timed CPU baseline; never linked into the product).
 *
 * Restates, for constant sound speed:
 *   gb/gb_solvers.py:356-422  solve_hom_diag (x(t), M(t) by Sherman-Morrison
 *                             :306-353, A(t) by :194-264)
 *   gb/core.py:16-36,171-191,194-329  compute_gaussian_beam_real (wrap,
 *                             safe angle, dense sum over beams, no cutoff)
 *   msgb_solver.py:612-619    mirror: every selected coefficient is
 *                             propagated with mode +1 and mode -1.
 * and the exact transpose of that sum down to the coefficients:
 *   g_b = sum_{t,s} 2 d(t,s) conj(K_b(t,s)),  contribution = 2 Re[c_b K_b].
 *
 * Beams are given once (positive branch); complex arrays are interleaved
 * (re, im).  Output rows are owned by one thread each, so results do not
 * depend on the thread count.
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

typedef double complex cplx;

typedef struct {
    double x[3];
    cplx M[3][3];
    cplx A;
} beam_state;

/* solve_hom_diag at one time for one beam (gb_solvers.py:356-422). */
static void hom_state(int d, const double *x0, const double *p0, const cplx *alpha,
                      cplx a0, double c0, double t, beam_state *st) {
    double n2 = 0.0;
    for (int i = 0; i < d; ++i) n2 += p0[i] * p0[i];
    double np_ = sqrt(n2);
    for (int i = 0; i < d; ++i) st->x[i] = x0[i] + c0 * (p0[i] / np_) * t;
    /* Sherman-Morrison, gb_solvers.py:330-353 */
    cplx Ainv[3], u[3], Ainv_u[3], vTAinv[3];
    for (int i = 0; i < d; ++i) {
        cplx Ad = 1.0 + c0 * t * alpha[i] / np_;
        Ainv[i] = 1.0 / Ad;
        u[i] = -c0 * t * p0[i] / (np_ * np_ * np_);
        Ainv_u[i] = Ainv[i] * u[i];
        vTAinv[i] = (p0[i] * alpha[i]) * Ainv[i];
    }
    cplx sc = 1.0;
    for (int j = 0; j < d; ++j) sc += vTAinv[j] * u[j];
    for (int i = 0; i < d; ++i)
        for (int j = 0; j < d; ++j) {
            cplx Y = (i == j ? Ainv[i] : 0.0) - Ainv_u[i] * vTAinv[j] / sc;
            st->M[i][j] = alpha[i] * Y;
        }
    /* amplitude, gb_solvers.py:194-264 */
    if (d == 3) {
        double p1 = p0[0] * p0[0], p2 = p0[1] * p0[1], p3 = p0[2] * p0[2];
        cplx a1 = alpha[0], a2 = alpha[1], a3 = alpha[2];
        double tsc = c0 * t / (n2 * n2);
        cplx t1 = c0 * a2 * a3 * t + (a2 + a3) * np_;
        cplx t2 = c0 * a1 * a3 * t + (a1 + a3) * np_;
        cplx t3 = c0 * a1 * a2 * t + (a1 + a2) * np_;
        cplx den = 1.0 + tsc * (p1 * t1 + p2 * t2 + p3 * t3);
        st->A = a0 / csqrt(den);
    } else {
        cplx ap = 0.0;
        for (int i = 0; i < d; ++i) ap += p0[i] * p0[i] * alpha[d - 1 - i];
        ap /= np_ * np_ * np_;
        if (d == 2)
            st->A = a0 / csqrt(1.0 + c0 * t * ap);
        else
            st->A = a0;
    }
}

static double pymod(double a, double b) {
    double r = fmod(a, b);
    if (r != 0.0 && ((r < 0.0) != (b < 0.0))) r += b;
    return r;
}

/* Complex exponent w*(p.D + D^T M D / 2) for one sensor (gb/core.py:292-303). */
static void phase_terms(int d, const beam_state *st, const double *p0, const double *s,
                        const double *L, const int *per, double *phi, double *chi) {
    double D[3];
    for (int i = 0; i < d; ++i) {
        double xi = per[i] ? pymod(st->x[i], L[i]) : st->x[i];
        double di = s[i] - xi;
        if (per[i]) di = di - L[i] * nearbyint(di / L[i]);
        D[i] = di;
    }
    double lin = 0.0, qr = 0.0, qi = 0.0;
    for (int i = 0; i < d; ++i) lin += D[i] * p0[i];
    for (int i = 0; i < d; ++i)
        for (int j = 0; j < d; ++j) {
            qr += D[i] * creal(st->M[i][j]) * D[j];
            qi += D[i] * cimag(st->M[i][j]) * D[j];
        }
    *phi = lin + 0.5 * qr;
    *chi = 0.5 * qi;
}

static double safe_angle(cplx z) {
    double re = creal(z), im = cimag(z);
    if (re == 0.0 && im == 0.0) re = 1e-12;
    return atan2(im, re);
}

/* Dense forward: out[t*ns + s] = sum over beams and both modes. */
int oracle_sum_hom(int d, int64_t n, const double *x0, const double *p0, const double *alpha,
                   const double *a0, const double *omega, double c, int64_t nt,
                   const double *ts, int64_t ns, const double *sens, const double *L,
                   const int *per, double *out) {
    if (d < 1 || d > 3) return 1;
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t t = 0; t < nt; ++t) {
        double *row = out + t * ns;
        for (int64_t s = 0; s < ns; ++s) row[s] = 0.0;
        for (int64_t b = 0; b < 2 * n; ++b) {
            int64_t j = b < n ? b : b - n;
            double c0 = b < n ? c : -c;
            cplx al[3];
            for (int i = 0; i < d; ++i) al[i] = alpha[2 * (j * d + i)] + I * alpha[2 * (j * d + i) + 1];
            beam_state st;
            hom_state(d, x0 + j * d, p0 + j * d, al, a0[2 * j] + I * a0[2 * j + 1], c0, ts[t], &st);
            double amp = 2.0 * cabs(st.A), ang = safe_angle(st.A), w = omega[j];
            for (int64_t s = 0; s < ns; ++s) {
                double phi, chi;
                phase_terms(d, &st, p0 + j * d, sens + s * d, L, per, &phi, &chi);
                row[s] += amp * cos(w * phi + ang) * exp(-w * chi);
            }
        }
    }
    return 0;
}

/* Exact transpose to the coefficients: g_j = sum_modes sum_{t,s} 2 d conj(K). a0 is the
 * unit amplitude (without the coefficient); g is interleaved complex (n). */
int oracle_adj_hom(int d, int64_t n, const double *x0, const double *p0, const double *alpha,
                   const double *a0, const double *omega, double c, int64_t nt,
                   const double *ts, int64_t ns, const double *sens, const double *L,
                   const int *per, const double *data, double *g) {
    if (d < 1 || d > 3) return 1;
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t j = 0; j < n; ++j) {
        cplx acc = 0.0;
        cplx al[3];
        for (int i = 0; i < d; ++i) al[i] = alpha[2 * (j * d + i)] + I * alpha[2 * (j * d + i) + 1];
        for (int m = 0; m < 2; ++m) {
            double c0 = m == 0 ? c : -c;
            for (int64_t t = 0; t < nt; ++t) {
                beam_state st;
                hom_state(d, x0 + j * d, p0 + j * d, al, a0[2 * j] + I * a0[2 * j + 1], c0, ts[t], &st);
                double w = omega[j];
                cplx ca = conj(st.A);
                const double *drow = data + t * ns;
                for (int64_t s = 0; s < ns; ++s) {
                    double phi, chi;
                    phase_terms(d, &st, p0 + j * d, sens + s * d, L, per, &phi, &chi);
                    double e = exp(-w * chi);
                    acc += 2.0 * drow[s] * ca * (cos(w * phi) - I * sin(w * phi)) * e;
                }
            }
        }
        g[2 * j] = creal(acc);
        g[2 * j + 1] = cimag(acc);
    }
    return 0;
}
