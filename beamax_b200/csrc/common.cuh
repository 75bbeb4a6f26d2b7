// Shared helpers for libmsgb: status handling, complex arithmetic, beam
// propagation in closed form (solve_hom_diag, beamax gb/gb_solvers.py:306-422).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>
#include <cstdio>
#include <string>

#include "../../include/msgb.h"

namespace msgb {

void set_error(const char *fmt, ...);
int fail(int code, const char *fmt, ...);
int check_launch(const char *what);

inline cudaStream_t as_stream(msgb_stream_t s) { return reinterpret_cast<cudaStream_t>(s); }

constexpr int kMaxDim = 3;

// ---------------------------------------------------------------- complex
struct cd {
    double re, im;
};

__host__ __device__ __forceinline__ cd mk(double r, double i) { return cd{r, i}; }
__host__ __device__ __forceinline__ cd operator+(cd a, cd b) { return cd{a.re + b.re, a.im + b.im}; }
__host__ __device__ __forceinline__ cd operator-(cd a, cd b) { return cd{a.re - b.re, a.im - b.im}; }
__host__ __device__ __forceinline__ cd operator*(cd a, cd b) {
    return cd{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
__host__ __device__ __forceinline__ cd operator*(double s, cd a) { return cd{s * a.re, s * a.im}; }
__host__ __device__ __forceinline__ cd conjc(cd a) { return cd{a.re, -a.im}; }
__device__ __forceinline__ cd divc(cd a, cd b) {
    // Smith's algorithm for a / b.
    if (fabs(b.re) >= fabs(b.im)) {
        double r = b.im / b.re, den = b.re + b.im * r;
        return cd{(a.re + a.im * r) / den, (a.im - a.re * r) / den};
    }
    double r = b.re / b.im, den = b.re * r + b.im;
    return cd{(a.re * r + a.im) / den, (a.im * r - a.re) / den};
}
// Principal square root (branch cut on the negative real axis).
__device__ __forceinline__ cd sqrtc(cd z) {
    double m = hypot(z.re, z.im);
    if (m == 0.0) return cd{0.0, 0.0};
    double r = sqrt(0.5 * (m + fabs(z.re)));
    if (z.re >= 0.0) return cd{r, z.im / (2.0 * r)};
    return cd{fabs(z.im) / (2.0 * r), copysign(r, z.im)};
}

// ---------------------------------------------------------------- beams
// Beam state at one time in closed form: centre x, complex Hessian M (packed
// symmetric, xx, xy, xz, yy, yz, zz order for D = 3; xx, xy, yy for D = 2; xx
// for D = 1) and complex amplitude A.  Restates gb_solvers.py:306-353
// (Sherman-Morrison) and :194-264 (amplitude), with c0 = mode * c.
template <int D>
struct HomState {
    double x[D];
    cd M[D * (D + 1) / 2];
    cd A;
};

template <int D>
__device__ __forceinline__ int sym_index(int i, int j) {
    if (i > j) {
        int t = i;
        i = j;
        j = t;
    }
    if (D == 1) return 0;
    if (D == 2) return i == 0 ? j : 2;
    // D == 3: (0,0)0 (0,1)1 (0,2)2 (1,1)3 (1,2)4 (2,2)5
    return i == 0 ? j : (i == 1 ? 2 + j : 5);
}

template <int D>
__device__ __forceinline__ void hom_state(const double *x0, const double *p0, const cd *alpha,
                                          cd a0, double c0, double t, HomState<D> &st) {
    double n2 = 0.0;
#pragma unroll
    for (int i = 0; i < D; ++i) n2 += p0[i] * p0[i];
    const double np = sqrt(n2);
#pragma unroll
    for (int i = 0; i < D; ++i) st.x[i] = x0[i] + c0 * (p0[i] / np) * t;
    cd Ainv[D], Ainv_u[D], vTAinv[D];
    double u[D];
    const double np3 = np * np * np;
#pragma unroll
    for (int i = 0; i < D; ++i) {
        cd Ad = cd{1.0, 0.0} + (c0 * t / np) * alpha[i];
        Ainv[i] = divc(cd{1.0, 0.0}, Ad);
        u[i] = -c0 * t * p0[i] / np3;
        Ainv_u[i] = u[i] * Ainv[i];
        vTAinv[i] = p0[i] * (alpha[i] * Ainv[i]);
    }
    cd sc = cd{1.0, 0.0};
#pragma unroll
    for (int j = 0; j < D; ++j) sc = sc + u[j] * vTAinv[j];
#pragma unroll
    for (int i = 0; i < D; ++i) {
#pragma unroll
        for (int j = i; j < D; ++j) {
            cd Y = divc(Ainv_u[i] * vTAinv[j], sc);
            Y = cd{-Y.re, -Y.im};
            if (i == j) Y = Y + Ainv[i];
            st.M[sym_index<D>(i, j)] = alpha[i] * Y;
        }
    }
    if (D == 3) {
        const double p1 = p0[0] * p0[0], p2 = p0[1] * p0[1], p3 = p0[2 % D] * p0[2 % D];
        const cd a1 = alpha[0], a2 = alpha[1 % D], a3 = alpha[2 % D];
        const double tsc = c0 * t / (n2 * n2);
        cd t1 = (c0 * t) * (a2 * a3) + np * (a2 + a3);
        cd t2 = (c0 * t) * (a1 * a3) + np * (a1 + a3);
        cd t3 = (c0 * t) * (a1 * a2) + np * (a1 + a2);
        cd den = cd{1.0, 0.0} + tsc * (p1 * t1 + p2 * t2 + p3 * t3);
        st.A = divc(a0, sqrtc(den));
    } else if (D == 2) {
        cd ap = p0[0] * p0[0] * alpha[1 % D] + p0[1 % D] * p0[1 % D] * alpha[0];
        ap = (1.0 / np3) * ap;
        st.A = divc(a0, sqrtc(cd{1.0, 0.0} + (c0 * t) * ap));
    } else {
        st.A = a0;
    }
}

__host__ __device__ __forceinline__ double pymod(double a, double b) {
    double r = fmod(a, b);
    if (r != 0.0 && ((r < 0.0) != (b < 0.0))) r += b;
    return r;
}

// Angle of A with the (eps, 0) substitution for exact zero (gb/core.py:171-191).
__device__ __forceinline__ double safe_angle(cd z) {
    double re = z.re;
    if (z.re == 0.0 && z.im == 0.0) re = 1e-12;
    return atan2(z.im, re);
}

// Problem parameters copied by value into kernels.
struct ProbArgs {
    int nd;
    int periodic[3];
    double L[3];
    double c;
    int64_t nt, ns;
    const double *ts;
    const double *sensors;
};

struct BeamArgs {
    int64_t n;
    const double *x0, *p0, *alpha, *a0, *omega;
    int modes;  // 0 both branches, 1 only mode +1, 2 only mode -1
};

__host__ __device__ __forceinline__ bool mode_on(int modes, int m) { return modes == 0 || modes == m + 1; }

int validate_problem(const msgb_problem *p);
int validate_beams(const msgb_problem *p, const msgb_beam_set *b);
ProbArgs to_args(const msgb_problem *p);
BeamArgs to_args(const msgb_beam_set *b);

}  // namespace msgb
