// Shared by the beam ODE (rk4.cu) and the trajectory surrogate (surrogate.cu):
// the sound speed interpolant with its derivatives, the beam state, and the
// writer of trajectory records (FP64 records, FP32 summation records, and the
// per-time-tile culling boxes) in the layout msgb_trajectories documents.
#pragma once

#include "common.cuh"

namespace msgb {
namespace {

struct MediumArgs {
    int kind, boundary;
    int n[3];
    double spacing[3], origin[3];
    double inv_spacing[3];  // 1 / spacing (multiplications instead of FP64 divisions)
    const double *coeffs;
    double c, lam;
    const float *coeffs32;  // (coeffs - c_ref) in FP32, or nullptr
    double c_ref;
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

// Tap k of the `taps` consecutive taps starting at lo: inside the grid (the
// usual case) the index itself, else the boundary rule.
__device__ __forceinline__ int tap_index(int lo, int k, int taps, int n, int boundary) {
    return (lo >= 0 && lo + taps <= n) ? lo + k : map_index(lo + k, n, boundary);
}

// c, grad c (D), hess c (D x D, row-major) at x, for a medium of kind KIND
// (the tap count and the weights are then compile-time constants).
template <int D, int KIND>
__device__ __forceinline__ void speed_eval_k(const MediumArgs &m, const double *x, double &c, double *g, double *H) {
    if (KIND == MSGB_MEDIUM_CONSTANT) {
        c = m.c;
#pragma unroll
        for (int i = 0; i < D; ++i) {
            g[i] = 0.0;
#pragma unroll
            for (int k = 0; k < D; ++k) H[i * D + k] = 0.0;
        }
        return;
    }
    constexpr bool cubic = KIND == MSGB_MEDIUM_BSPLINE3;
    constexpr int taps = cubic ? 4 : 2;
    constexpr int off0 = cubic ? -1 : 0;
    double w[D][4], d1[D][4], d2[D][4];
    int idx[D][4];
#pragma unroll
    for (int a = 0; a < D; ++a) {
        const double u = (x[a] - m.origin[a]) * m.inv_spacing[a];
        const double fl = floor(u);
        const double t = u - fl;
        const int i0 = (int)fl;
        if (cubic) {
            // 6 x the B-spline weights (the factors 1/6 are applied to the
            // sums at the end: no FP64 division per weight)
            const double omt = 1.0 - t, t2 = t * t, t3 = t2 * t;
            w[a][0] = omt * omt * omt;
            w[a][1] = 3.0 * t3 - 6.0 * t2 + 4.0;
            w[a][2] = -3.0 * t3 + 3.0 * t2 + 3.0 * t + 1.0;
            w[a][3] = t3;
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
#pragma unroll
        for (int k = 0; k < taps; ++k) idx[a][k] = tap_index(i0 + off0, k, taps, m.n[a], m.boundary);
    }
    // Separable reduction, last axis first: the tensor-product weights factor,
    // so the value, gradient and Hessian need 3 sums per line of the last
    // axis instead of D^2 products per grid corner.
    double cc = 0.0, gg[D], hh[D][D];
#pragma unroll
    for (int i = 0; i < D; ++i) {
        gg[i] = 0.0;
#pragma unroll
        for (int k = 0; k < D; ++k) hh[i][k] = 0.0;
    }
    if (D == 1) {
#pragma unroll
        for (int k = 0; k < taps; ++k) {
            const double v = __ldg(m.coeffs + idx[0][k]);
            cc = fma(w[0][k], v, cc);
            gg[0] = fma(d1[0][k], v, gg[0]);
            hh[0][0] = fma(d2[0][k], v, hh[0][0]);
        }
    } else if (D == 2) {
        const int L = D - 1;  // last axis
#pragma unroll
        for (int i = 0; i < taps; ++i) {
            const double *row = m.coeffs + (int64_t)idx[0][i] * m.n[L];
            double rw = 0.0, rd = 0.0, rdd = 0.0;
#pragma unroll
            for (int k = 0; k < taps; ++k) {
                const double v = __ldg(row + idx[L][k]);
                rw = fma(w[L][k], v, rw);
                rd = fma(d1[L][k], v, rd);
                rdd = fma(d2[L][k], v, rdd);
            }
            cc = fma(w[0][i], rw, cc);
            gg[0] = fma(d1[0][i], rw, gg[0]);
            gg[L] = fma(w[0][i], rd, gg[L]);
            hh[0][0] = fma(d2[0][i], rw, hh[0][0]);
            hh[0][L] = fma(d1[0][i], rd, hh[0][L]);
            hh[L][L] = fma(w[0][i], rdd, hh[L][L]);
        }
    } else {
        const int Y = 1 % D, Z = 2 % D;
#pragma unroll
        for (int i = 0; i < taps; ++i) {
            double tw = 0.0, ty = 0.0, tyy = 0.0, tz = 0.0, tyz = 0.0, tzz = 0.0;
#pragma unroll
            for (int j = 0; j < taps; ++j) {
                const double *line = m.coeffs + ((int64_t)idx[0][i] * m.n[Y] + idx[Y][j]) * m.n[Z];
                double sw = 0.0, sd = 0.0, sdd = 0.0;
#pragma unroll
                for (int k = 0; k < taps; ++k) {
                    const double v = __ldg(line + idx[Z][k]);
                    sw = fma(w[Z][k], v, sw);
                    sd = fma(d1[Z][k], v, sd);
                    sdd = fma(d2[Z][k], v, sdd);
                }
                tw = fma(w[Y][j], sw, tw);
                ty = fma(d1[Y][j], sw, ty);
                tyy = fma(d2[Y][j], sw, tyy);
                tz = fma(w[Y][j], sd, tz);
                tyz = fma(d1[Y][j], sd, tyz);
                tzz = fma(w[Y][j], sdd, tzz);
            }
            cc = fma(w[0][i], tw, cc);
            gg[0] = fma(d1[0][i], tw, gg[0]);
            gg[Y] = fma(w[0][i], ty, gg[Y]);
            gg[Z] = fma(w[0][i], tz, gg[Z]);
            hh[0][0] = fma(d2[0][i], tw, hh[0][0]);
            hh[0][Y] = fma(d1[0][i], ty, hh[0][Y]);
            hh[0][Z] = fma(d1[0][i], tz, hh[0][Z]);
            hh[Y][Y] = fma(w[0][i], tyy, hh[Y][Y]);
            hh[Y][Z] = fma(w[0][i], tyz, hh[Y][Z]);
            hh[Z][Z] = fma(w[0][i], tzz, hh[Z][Z]);
        }
    }
    // Cubic weights were 6 x the true ones: a sum whose terms carry the plain
    // weight of q axes is 6^q too large (value: D axes; gradient: D - 1;
    // diagonal Hessian: D - 1; mixed Hessian: D - 2).
    constexpr double s6 = cubic ? 1.0 / 6.0 : 1.0;
    constexpr double sv = D == 1 ? s6 : (D == 2 ? s6 * s6 : s6 * s6 * s6);
    constexpr double sg = D == 1 ? 1.0 : (D == 2 ? s6 : s6 * s6);
    constexpr double sm = D == 3 ? s6 : 1.0;
    c = cc * sv;
#pragma unroll
    for (int a = 0; a < D; ++a) {
        g[a] = gg[a] * (sg * m.inv_spacing[a]);
#pragma unroll
        for (int b = 0; b < D; ++b) {
            const double hv = a <= b ? hh[a][b] : hh[b][a];
            H[a * D + b] = hv * ((a == b ? sg : sm) * m.inv_spacing[a] * m.inv_spacing[b]);
        }
    }
}

// The same in FP32 for the FP32 path: the fractional position is formed in
// FP64 and rounded, the B-spline weights and tap sums run in FP32 on
// (coefficient - c_ref) values centred on tap (1, 1[, 1]) of the stencil (the
// weights of every derivative sum to zero, so the centring leaves the
// gradient and Hessian unchanged and keeps their sums free of cancellation;
// the value gets the centre back), and the results return to FP64 with c_ref.
template <int D, int KIND>
__device__ __forceinline__ void speed_eval_f32(const MediumArgs &m, const double *x, double &c, double *g,
                                               double *H) {
    constexpr bool cubic = KIND == MSGB_MEDIUM_BSPLINE3;
    constexpr int taps = cubic ? 4 : 2;
    constexpr int off0 = cubic ? -1 : 0;
    constexpr int ctr = cubic ? 1 : 0;  // the tap at the cell's lower corner
    float w[D][4], d1[D][4], d2[D][4];
    int idx[D][4];
#pragma unroll
    for (int a = 0; a < D; ++a) {
        const double u = (x[a] - m.origin[a]) * m.inv_spacing[a];
        const double fl = floor(u);
        const float t = (float)(u - fl);
        const int i0 = (int)fl;
        if (cubic) {
            const float omt = 1.0f - t, t2 = t * t, t3 = t2 * t;
            w[a][0] = omt * omt * omt;
            w[a][1] = fmaf(3.0f, t3, fmaf(-6.0f, t2, 4.0f));
            w[a][2] = fmaf(-3.0f, t3, fmaf(3.0f, t2, fmaf(3.0f, t, 1.0f)));
            w[a][3] = t3;
            d1[a][0] = -0.5f * omt * omt;
            d1[a][1] = fmaf(1.5f, t2, -2.0f * t);
            d1[a][2] = fmaf(-1.5f, t2, t + 0.5f);
            d1[a][3] = 0.5f * t2;
            d2[a][0] = omt;
            d2[a][1] = fmaf(3.0f, t, -2.0f);
            d2[a][2] = fmaf(-3.0f, t, 1.0f);
            d2[a][3] = t;
        } else {
            w[a][0] = 1.0f - t;
            w[a][1] = t;
            d1[a][0] = -1.0f;
            d1[a][1] = 1.0f;
            d2[a][0] = d2[a][1] = 0.0f;
            w[a][2] = w[a][3] = d1[a][2] = d1[a][3] = d2[a][2] = d2[a][3] = 0.0f;
        }
#pragma unroll
        for (int k = 0; k < taps; ++k) idx[a][k] = tap_index(i0 + off0, k, taps, m.n[a], m.boundary);
    }
    float cc = 0.0f, gg[D], hh[D][D];
#pragma unroll
    for (int i = 0; i < D; ++i) {
        gg[i] = 0.0f;
#pragma unroll
        for (int k = 0; k < D; ++k) hh[i][k] = 0.0f;
    }
    float vc;
    if (D == 1) {
        vc = __ldg(m.coeffs32 + idx[0][ctr]);
#pragma unroll
        for (int k = 0; k < taps; ++k) {
            const float v = __ldg(m.coeffs32 + idx[0][k]) - vc;
            cc = fmaf(w[0][k], v, cc);
            gg[0] = fmaf(d1[0][k], v, gg[0]);
            hh[0][0] = fmaf(d2[0][k], v, hh[0][0]);
        }
    } else if (D == 2) {
        const int L = D - 1;
        vc = __ldg(m.coeffs32 + (int64_t)idx[0][ctr] * m.n[L] + idx[L][ctr]);
#pragma unroll
        for (int i = 0; i < taps; ++i) {
            const float *row = m.coeffs32 + (int64_t)idx[0][i] * m.n[L];
            float rw = 0.0f, rd = 0.0f, rdd = 0.0f;
#pragma unroll
            for (int k = 0; k < taps; ++k) {
                const float v = __ldg(row + idx[L][k]) - vc;
                rw = fmaf(w[L][k], v, rw);
                rd = fmaf(d1[L][k], v, rd);
                rdd = fmaf(d2[L][k], v, rdd);
            }
            cc = fmaf(w[0][i], rw, cc);
            gg[0] = fmaf(d1[0][i], rw, gg[0]);
            gg[L] = fmaf(w[0][i], rd, gg[L]);
            hh[0][0] = fmaf(d2[0][i], rw, hh[0][0]);
            hh[0][L] = fmaf(d1[0][i], rd, hh[0][L]);
            hh[L][L] = fmaf(w[0][i], rdd, hh[L][L]);
        }
    } else {
        const int Y = 1 % D, Z = 2 % D;
        vc = __ldg(m.coeffs32 + ((int64_t)idx[0][ctr] * m.n[Y] + idx[Y][ctr]) * m.n[Z] + idx[Z][ctr]);
#pragma unroll
        for (int i = 0; i < taps; ++i) {
            float tw = 0.0f, ty = 0.0f, tyy = 0.0f, tz = 0.0f, tyz = 0.0f, tzz = 0.0f;
#pragma unroll
            for (int j = 0; j < taps; ++j) {
                const float *line = m.coeffs32 + ((int64_t)idx[0][i] * m.n[Y] + idx[Y][j]) * m.n[Z];
                float sw = 0.0f, sd = 0.0f, sdd = 0.0f;
#pragma unroll
                for (int k = 0; k < taps; ++k) {
                    const float v = __ldg(line + idx[Z][k]) - vc;
                    sw = fmaf(w[Z][k], v, sw);
                    sd = fmaf(d1[Z][k], v, sd);
                    sdd = fmaf(d2[Z][k], v, sdd);
                }
                tw = fmaf(w[Y][j], sw, tw);
                ty = fmaf(d1[Y][j], sw, ty);
                tyy = fmaf(d2[Y][j], sw, tyy);
                tz = fmaf(w[Y][j], sd, tz);
                tyz = fmaf(d1[Y][j], sd, tyz);
                tzz = fmaf(w[Y][j], sdd, tzz);
            }
            cc = fmaf(w[0][i], tw, cc);
            gg[0] = fmaf(d1[0][i], tw, gg[0]);
            gg[Y] = fmaf(w[0][i], ty, gg[Y]);
            gg[Z] = fmaf(w[0][i], tz, gg[Z]);
            hh[0][0] = fmaf(d2[0][i], tw, hh[0][0]);
            hh[0][Y] = fmaf(d1[0][i], ty, hh[0][Y]);
            hh[0][Z] = fmaf(d1[0][i], tz, hh[0][Z]);
            hh[Y][Y] = fmaf(w[0][i], tyy, hh[Y][Y]);
            hh[Y][Z] = fmaf(w[0][i], tyz, hh[Y][Z]);
            hh[Z][Z] = fmaf(w[0][i], tzz, hh[Z][Z]);
        }
    }
    constexpr double s6 = cubic ? 1.0 / 6.0 : 1.0;
    constexpr double sv = D == 1 ? s6 : (D == 2 ? s6 * s6 : s6 * s6 * s6);
    constexpr double sg = D == 1 ? 1.0 : (D == 2 ? s6 : s6 * s6);
    constexpr double sm = D == 3 ? s6 : 1.0;
    // the value's weights sum to 1: the centre comes back in FP64
    c = m.c_ref + (double)vc + (double)cc * sv;
#pragma unroll
    for (int a = 0; a < D; ++a) {
        g[a] = (double)gg[a] * (sg * m.inv_spacing[a]);
#pragma unroll
        for (int b = 0; b < D; ++b) {
            const double hv = a <= b ? (double)hh[a][b] : (double)hh[b][a];
            H[a * D + b] = hv * ((a == b ? sg : sm) * m.inv_spacing[a] * m.inv_spacing[b]);
        }
    }
}

// The same for a medium kind known only at run time.
template <int D>
__device__ void speed_eval(const MediumArgs &m, const double *x, double &c, double *g, double *H) {
    switch (m.kind) {
        case MSGB_MEDIUM_CONSTANT: speed_eval_k<D, MSGB_MEDIUM_CONSTANT>(m, x, c, g, H); break;
        case MSGB_MEDIUM_LINEAR: speed_eval_k<D, MSGB_MEDIUM_LINEAR>(m, x, c, g, H); break;
        default: speed_eval_k<D, MSGB_MEDIUM_BSPLINE3>(m, x, c, g, H); break;
    }
}

template <int D>
struct State {
    double x[D], p[D];
    cd M[D][D];
    cd A;
};

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
    // compact FP32 store (pool != nullptr): see msgb_trajectories
    int32_t *slot = nullptr;
    void *pool = nullptr;
    float *pool_cull = nullptr;
    int64_t pool_blocks = 0;
    unsigned long long *pool_next = nullptr;
    const float *boxes = nullptr;
    int64_t n_boxes = 0;
    float live_cutoff = 0.0f;
};

// Host: the compact-store fields of a msgb_trajectories descriptor.
inline void set_compact(TrajArgs &T, const msgb_trajectories *t) {
    T.slot = t->slot;
    T.pool = t->pool;
    T.pool_cull = t->pool_cull;
    T.pool_blocks = t->pool_blocks;
    T.pool_next = t->pool_next;
    T.boxes = t->live_boxes;
    T.n_boxes = t->n_boxes;
    T.live_cutoff = (float)t->live_cutoff;
}

inline int check_compact(const msgb_trajectories *t, int ndim) {
    if (!t->pool) return MSGB_OK;
    if (t->rec32) return fail(MSGB_ERR_ARG, "trajectories: rec32 and a compact pool are exclusive");
    if (!t->slot || !t->pool_cull || !t->pool_next || t->pool_blocks < 1)
        return fail(MSGB_ERR_ARG, "trajectories: compact store needs slot, pool_cull, pool_next and pool_blocks > 0");
    if (t->n_boxes < 0 || (t->n_boxes > 0 && !t->live_boxes))
        return fail(MSGB_ERR_ARG, "trajectories: live_boxes is NULL");
    if (!(t->live_cutoff >= 0.0)) return fail(MSGB_ERR_ARG, "trajectories: live_cutoff must be >= 0");
    (void)ndim;
    return MSGB_OK;
}


// Writes the records of one beam (index bl within the chunk) at every time k,
// and the culling box of each time tile as its last time is written.
template <int D>
struct RecordWriter {
    static constexpr int S = D * (D + 1) / 2;
    static constexpr int NR64 = 2 * D + 2 * D * D + 2;
    const ProbArgs &P;
    const TrajArgs &T;
    int64_t bl;
    double w;
    int tt_len;
    float lo[D], hi[D];
    double lmin = 1e300;
    bool bad = false;
    // compact store: this lane's block for the current time tile (-1: none
    // taken yet; kept across beams when a dead tile did not use it)
    int64_t blk = -1;

    __device__ RecordWriter(const ProbArgs &P_, const TrajArgs &T_, int64_t bl_, double w_, int tt_len_)
        : P(P_), T(T_), bl(bl_), w(w_), tt_len(tt_len_) {
#pragma unroll
        for (int i = 0; i < D; ++i) lo[i] = 3.4e38f, hi[i] = -3.4e38f;
    }

    // Start the records of another beam of the same chunk.
    __device__ void reset(int64_t bl_, double w_) {
        bl = bl_;
        w = w_;
        lmin = 1e300;
        bad = false;
#pragma unroll
        for (int i = 0; i < D; ++i) lo[i] = 3.4e38f, hi[i] = -3.4e38f;
    }

    // `failed`: the state is not trustworthy from here on (never culled).
    __device__ void put(int64_t k, const State<D> &y, bool failed) {
        bad |= failed;
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
        const int kk_tile = (int)(k % tt_len);
        char *rec32_base = nullptr;
        if (T.pool) {
            if (kk_tile == 0 && blk < 0) blk = (int64_t)atomicAdd(T.pool_next, 1ULL);
            if (blk >= 0 && blk < T.pool_blocks)
                rec32_base = (char *)T.pool + (blk * tt_len + kk_tile) * (int64_t)(16 * D + 8 * S + 8);
        } else if (T.rec32) {
            rec32_base = (char *)T.rec32 + (k * T.nb + bl) * (int64_t)(16 * D + 8 * S + 8);
        }
        if (rec32_base) {
            // layout of the FP32 summation's BeamTime<D> record
            char *base = rec32_base;
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
            // arg A and 2|A| are stored as floats: FP32 arithmetic on the
            // rounded components gives them to FP32 precision
            const float are = (float)y.A.re, aim = (float)y.A.im;
            f[2 * S] = atan2f(aim, (are == 0.0f && aim == 0.0f) ? 1e-12f : are);
            f[2 * S + 1] = 2.0f * hypotf(are, aim);
        }
        if (T.cull || T.pool) {
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
                float box[2 * D + 1];
#pragma unroll
                for (int i = 0; i < D; ++i) {
                    // periodic axes and non-finite states are never culled
                    const bool open = P.periodic[i] || bad;
                    box[i] = open ? -3.4e38f : lo[i];
                    box[D + i] = open ? 3.4e38f : hi[i];
                }
                box[2 * D] = bad ? 0.0f : (float)fmax(0.0, 0.5 * w * lmin * (1.0 - 1e-6));
                if (T.pool) {
                    // live: within the cutoff of some sensor tile (the summation's
                    // own test, with the cutoff widened by 1e-4 so that every
                    // tile the summation keeps is stored)
                    bool live = bad || T.n_boxes == 0;
                    for (int64_t q = 0; q < T.n_boxes && !live; ++q) {
                        const float *tb = T.boxes + q * 2 * D;
                        float d2 = 0.0f;
#pragma unroll
                        for (int i = 0; i < D; ++i) {
                            const float gap = fmaxf(0.0f, fmaxf(tb[i] - box[D + i], box[i] - tb[D + i]));
                            d2 = fmaf(gap, gap, d2);
                        }
                        live = box[2 * D] * d2 * 0.999f <= T.live_cutoff * 1.0001f;
                    }
                    int32_t *sl = T.slot + (k / tt_len) * T.nb + bl;
                    if (live && blk >= 0 && blk < T.pool_blocks) {
                        *sl = (int32_t)blk;
                        float *c = T.pool_cull + blk * (2 * D + 1);
#pragma unroll
                        for (int i = 0; i < 2 * D + 1; ++i) c[i] = box[i];
                        blk = -1;  // the block belongs to this tile now
                    } else {
                        *sl = -1;  // dead tile (or pool exhausted): the block is reused
                    }
                } else {
                    float *c = T.cull + ((k / tt_len) * T.nb + bl) * (2 * D + 1);
#pragma unroll
                    for (int i = 0; i < 2 * D + 1; ++i) c[i] = box[i];
                }
            }
        }
    }
};

// Host: medium description -> kernel arguments (MSGB_OK or an error code).
inline int medium_args(const msgb_problem *prob, const msgb_medium *med, MediumArgs &M) {
    if (!med) return fail(MSGB_ERR_ARG, "medium is NULL");
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
    M = MediumArgs{};
    M.kind = med->kind;
    M.boundary = med->boundary;
    for (int a = 0; a < 3; ++a) {
        M.n[a] = med->n[a];
        M.spacing[a] = med->spacing[a];
        M.origin[a] = med->origin[a];
    }
    for (int a = 0; a < 3; ++a) M.inv_spacing[a] = 1.0 / M.spacing[a];
    M.coeffs = med->coeffs;
    M.c = med->c;
    M.lam = med->lam;
    M.coeffs32 = med->coeffs32;
    M.c_ref = med->c_ref;
    return MSGB_OK;
}

}  // namespace
}  // namespace msgb
