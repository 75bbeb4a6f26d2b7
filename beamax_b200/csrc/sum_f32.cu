// FP32 Gaussian-beam summation with Gaussian-cutoff culling, and its transpose.
//
// Same operator as compute_gaussian_beam_real (beamax gb/core.py:194-329)
// with solve_hom_diag (gb/gb_solvers.py:356-422):
//   out(t, s) = sum_b Re[z_b(t, s)],  z = 2|A| exp(i theta - chi),
//   theta = w (p.D + D^T Re M D / 2) + arg A,  chi = w D^T Im M D / 2,
//   D = s - x_b(t).
//
// Precision plan
//  * Sensors are grouped into tiles of TS sensors, ordered so that tiles hold
//    straight, evenly spaced runs (coarse-cell Morton order, row-major inside a
//    cell).  Each tile has an FP64 anchor s0.  Per (beam, time) the large phase
//    w p.(s0 - x(t)) + arg A is formed in FP64 and reduced to [-pi, pi) before
//    it meets FP32; per sensor only w p.(s - s0) (bounded by the tile) is FP32.
//  * Along a run s_k = s_a + k h the exponent i theta - chi is a quadratic in k,
//    so z_{k+1} = z_k r_k, r_{k+1} = r_k q with r_0 = exp(a1 + a2), q =
//    exp(2 a2): two complex multiplies per sensor.  Every run starts with a
//    direct evaluation (MUFU sincos/exp after explicit range reduction) and
//    runs are at most GS sensors long, which bounds the recurrence's relative
//    error growth (~k^2 eps / 2 < 1e-5).
//  * Accumulation across beams is Kahan-compensated FP32.
// Culling: for a (beam, time tile, sensor tile) triple
//   chi >= (w/2) lambda_min(Im M(t)) |D|^2 >= (w/2) lam_lo(t_b) dist^2,
// lam_lo(t) = 1 / (1/beta_min + (c t/|p|)^2 beta_max): with M0 = i diag(beta),
// Im M(t) = (S + R S^-1 R)^-1, S = diag(1/beta), R = (c t/|p|) P_perp, which is
// Loewner-decreasing in |t|; dist is the gap between the bounding boxes of the
// centre's path over the time tile and of the sensor tile.  A triple is
// skipped when that bound exceeds `cutoff` e-folds.
#include <cub/cub.cuh>

#include <mutex>

#include "common.cuh"

namespace msgb {
namespace {

constexpr int TT = 32;               // times per tile (= lanes)
constexpr int GS = 16;               // sensors per warp group and maximal run length
constexpr int NW = 8;                // warps per CTA (forward)
constexpr int TS = GS * NW;          // sensors per tile
constexpr int THREADS = NW * 32;
constexpr int G = THREADS / TT;      // beams per record pass
static_assert(G % 2 == 0, "beams are evaluated in pairs");
constexpr float kTwoPi = 6.283185307179586f;
constexpr float kInvTwoPi = 0.15915494309189535f;

// Reduce an FP32 angle to [-pi, pi] (bounded inputs).
__device__ __forceinline__ float reduce_angle(float th) {
    const float k = rintf(th * kInvTwoPi);
    return fmaf(-k, kTwoPi, th);
}

struct cf {
    float re, im;
};
__device__ __forceinline__ cf cmul(cf a, cf b) {
    return cf{fmaf(a.re, b.re, -a.im * b.im), fmaf(a.re, b.im, a.im * b.re)};
}
__device__ __forceinline__ cf cdiv(cf a, cf b) {
    const float inv = __frcp_rn(fmaf(b.re, b.re, b.im * b.im));
    return cf{(a.re * b.re + a.im * b.im) * inv, (a.im * b.re - a.re * b.im) * inv};
}
__device__ __forceinline__ cf csqrtf_(cf z) {
    const float m = sqrtf(fmaf(z.re, z.re, z.im * z.im));
    if (m == 0.0f) return cf{0.0f, 0.0f};
    const float r = sqrtf(0.5f * (m + fabsf(z.re)));
    if (z.re >= 0.0f) return cf{r, z.im / (2.0f * r)};
    return cf{fabsf(z.im) / (2.0f * r), copysignf(r, z.im)};
}
#ifndef MSGB_F32X2
#define MSGB_F32X2 1
#endif
#if MSGB_F32X2
// Two complex numbers, component-packed, for the paired FP32 instructions of
// sm_100 (FFMA2 / FMUL2 / FADD2).  Each lane of a paired operation rounds
// exactly as the scalar instruction, so these produce the same bits as cmul
// and kahan_add applied to each half.
struct cf2 {
    float2 re, im;
};
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ cf2 cmul2(cf2 a, cf2 b) {
    return cf2{__ffma2_rn(a.re, b.re, neg2(__fmul2_rn(a.im, b.im))), __ffma2_rn(a.re, b.im, __fmul2_rn(a.im, b.re))};
}
__device__ __forceinline__ void kahan_add2(float2 &acc, float2 &cmp, float2 v) {
    const float2 y = __fadd2_rn(v, neg2(cmp));
    const float2 t = __fadd2_rn(acc, y);
    cmp = __fadd2_rn(__fadd2_rn(t, neg2(acc)), neg2(y));
    acc = t;
}
__device__ __forceinline__ cf2 pack2(cf a, cf b) { return cf2{make_float2(a.re, b.re), make_float2(a.im, b.im)}; }
#endif

// exp(x + i y) with y range-reduced first.
__device__ __forceinline__ cf cexpf_(float x, float y) {
    float s, c;
    __sincosf(reduce_angle(y), &s, &c);
    const float e = __expf(x);
    return cf{e * c, e * s};
}

template <int D>
struct Sym {
    static constexpr int S = D * (D + 1) / 2;
};

// Quadratic form with packed coefficients (off-diagonals already doubled).
template <int D>
__device__ __forceinline__ float quad(const float *c, const float *v) {
    float r = 0.0f;
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
        for (int k = i; k < D; ++k) r = fmaf(c[sym_index<D>(i, k)], v[i] * v[k], r);
    return r;
}
// 2 u^T C v for the same packed coefficients.
template <int D>
__device__ __forceinline__ float bilin2(const float *c, const float *u, const float *v) {
    float r = 0.0f;
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
        for (int k = i; k < D; ++k) {
            const float ck = c[sym_index<D>(i, k)];
            r = (i == k) ? fmaf(2.0f * ck, u[i] * v[i], r) : fmaf(ck, fmaf(u[i], v[k], u[k] * v[i]), r);
        }
    return r;
}

// Per (beam, time) evaluation record.
template <int D>
struct Rec {
    float d0[D];             // s0 - x(t)
    float wp[D];             // w p
    float q[Sym<D>::S];      // w/2 Re M (off-diagonals doubled)
    float p[Sym<D>::S];      // w/2 Im M (off-diagonals doubled)
    float th0;               // reduce(w p.(s0 - x(t)) + arg A)
    float amp;               // 2 |A(t)|
    static constexpr int NF = 2 * D + 2 * Sym<D>::S + 2;
};

// Tile-independent part of a record (the FP64 centre and the FP32 shape).
template <int D>
struct BeamTime {
    double x[D];
    double wp[D];
    float q[Sym<D>::S], p[Sym<D>::S];
    float ang, amp;
};

// Per selected coefficient culling data (mode independent).
template <int D>
struct Cull {
    float x0[D];
    float dir[D];   // p0 / |p0|
    float bmin, bmax, w, inv_np;
    int ok;         // 0: M0 not of the form i diag(beta) -> never culled
};

template <int D>
struct TileInfo {
    double s0[D];
    float lo[D], hi[D];
};

// Closed-form Hessian and amplitude in FP32 (gb_solvers.py:306-353, :194-264).
template <int D>
__device__ __forceinline__ void hom_mA_f32(const float *p0, const cf *al, cf a0, float c0t, cf *M, cf &A) {
    float n2 = 0.0f;
#pragma unroll
    for (int i = 0; i < D; ++i) n2 = fmaf(p0[i], p0[i], n2);
    const float np = sqrtf(n2);
    const float inv_np = 1.0f / np;
    const float np3 = n2 * np;
    cf Ainv[D], Ainv_u[D], vT[D];
    float u[D];
#pragma unroll
    for (int i = 0; i < D; ++i) {
        const float f = c0t * inv_np;
        cf Ad = cf{fmaf(f, al[i].re, 1.0f), f * al[i].im};
        Ainv[i] = cdiv(cf{1.0f, 0.0f}, Ad);
        u[i] = -c0t * p0[i] / np3;
        Ainv_u[i] = cf{u[i] * Ainv[i].re, u[i] * Ainv[i].im};
        cf t = cmul(al[i], Ainv[i]);
        vT[i] = cf{p0[i] * t.re, p0[i] * t.im};
    }
    cf sc = cf{1.0f, 0.0f};
#pragma unroll
    for (int j = 0; j < D; ++j) sc = cf{fmaf(u[j], vT[j].re, sc.re), fmaf(u[j], vT[j].im, sc.im)};
    const cf isc = cdiv(cf{1.0f, 0.0f}, sc);
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
        for (int j = i; j < D; ++j) {
            cf Y = cmul(cmul(Ainv_u[i], vT[j]), isc);
            Y = cf{-Y.re, -Y.im};
            if (i == j) Y = cf{Y.re + Ainv[i].re, Y.im + Ainv[i].im};
            M[sym_index<D>(i, j)] = cmul(al[i], Y);
        }
    if (D == 3) {
        const float p1 = p0[0] * p0[0], p2 = p0[1 % D] * p0[1 % D], p3 = p0[2 % D] * p0[2 % D];
        const cf a1 = al[0], a2 = al[1 % D], a3 = al[2 % D];
        const float tsc = c0t / (n2 * n2);
        auto term = [&](cf x, cf y) {
            cf xy = cmul(x, y);
            return cf{fmaf(c0t, xy.re, np * (x.re + y.re)), fmaf(c0t, xy.im, np * (x.im + y.im))};
        };
        cf t1 = term(a2, a3), t2 = term(a1, a3), t3 = term(a1, a2);
        cf s = cf{p1 * t1.re + p2 * t2.re + p3 * t3.re, p1 * t1.im + p2 * t2.im + p3 * t3.im};
        cf den = cf{fmaf(tsc, s.re, 1.0f), tsc * s.im};
        A = cdiv(a0, csqrtf_(den));
    } else if (D == 2) {
        cf ap = cf{(p0[0] * p0[0] * al[1 % D].re + p0[1 % D] * p0[1 % D] * al[0].re) / np3,
                   (p0[0] * p0[0] * al[1 % D].im + p0[1 % D] * p0[1 % D] * al[0].im) / np3};
        A = cdiv(a0, csqrtf_(cf{fmaf(c0t, ap.re, 1.0f), c0t * ap.im}));
    } else {
        A = a0;
    }
}

// Beam b in [0, 2n) (b >= n: mode -1) at time t, anchor-independent part.
template <int D>
__device__ __forceinline__ void beam_time(const ProbArgs &P, const BeamArgs &B, int64_t b, double t,
                                          BeamTime<D> &r) {
    const int64_t j = b < B.n ? b : b - B.n;
    const double c0 = b < B.n ? P.c : -P.c;
    double p0d[D], n2 = 0.0;
#pragma unroll
    for (int i = 0; i < D; ++i) {
        p0d[i] = B.p0[j * D + i];
        n2 += p0d[i] * p0d[i];
    }
    const double np = sqrt(n2);
    const double w = B.omega[j];
    float p0f[D];
    cf al[D];
#pragma unroll
    for (int i = 0; i < D; ++i) {
        double x = B.x0[j * D + i] + c0 * (p0d[i] / np) * t;
        if (P.periodic[i]) x = pymod(x, P.L[i]);
        r.x[i] = x;
        r.wp[i] = w * p0d[i];
        p0f[i] = (float)p0d[i];
        al[i] = cf{(float)B.alpha[2 * (j * D + i)], (float)B.alpha[2 * (j * D + i) + 1]};
    }
    cf M[Sym<D>::S], A;
    hom_mA_f32<D>(p0f, al, cf{(float)B.a0[2 * j], (float)B.a0[2 * j + 1]}, (float)(c0 * t), M, A);
    const float wf = (float)w;
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
        for (int k = i; k < D; ++k) {
            const int q = sym_index<D>(i, k);
            const float f = (i == k ? 0.5f : 1.0f) * wf;
            r.q[q] = f * M[q].re;
            r.p[q] = f * M[q].im;
        }
    float re = A.re;
    if (A.re == 0.0f && A.im == 0.0f) re = 1e-12f;
    r.ang = atan2f(A.im, re);
    r.amp = 2.0f * sqrtf(fmaf(A.re, A.re, A.im * A.im));
}

// Anchor-dependent completion of a record.
template <int D>
__device__ __forceinline__ void anchor(const ProbArgs &P, const BeamTime<D> &bt, const double *s0, Rec<D> &r) {
    double lin = 0.0;
#pragma unroll
    for (int i = 0; i < D; ++i) {
        double d0 = s0[i] - bt.x[i];
        if (P.periodic[i]) d0 -= P.L[i] * nearbyint(d0 / P.L[i]);
        r.d0[i] = (float)d0;
        r.wp[i] = (float)bt.wp[i];
        lin = fma(bt.wp[i], d0, lin);
    }
#pragma unroll
    for (int q = 0; q < Sym<D>::S; ++q) {
        r.q[q] = bt.q[q];
        r.p[q] = bt.p[q];
    }
    const double th = lin + (double)bt.ang;
    r.th0 = (float)(th - 6.283185307179586 * nearbyint(th * 0.15915494309189535));
    r.amp = bt.amp;
}

// Largest e-fold count the run recurrence may meet: at the seed (chi), in the
// first step's ratio and in the ratio's own step.  Beyond it the factors leave
// FP32's range (e^88) and the recurrence would produce 0 * inf; such runs are
// evaluated directly.  Only very narrow beams (e-fold width under about one
// sensor spacing over a 16-sensor run, e.g. after focusing in a
// heterogeneous medium) reach it.
constexpr float kRecurrenceEfolds = 60.0f;
// A run whose smallest exponent over its 16 sensors exceeds this many e-folds
// contributes below 4e-18 of the beam's amplitude and is skipped (only when
// culling is enabled, cutoff > 0).
constexpr float kNegligibleEfolds = 40.0f;

enum RunKind { kRunRecurrence = 0, kRunNegligible = 1, kRunDirect = 2 };

// Direct evaluation at a run start (seed): z, and the recurrence factors for
// the step h to the next sensor.  With `kind`, classifies the run of GS
// sensors (RunKind): the exponent along it is chi(k) = chi + B k + A k^2 with
// B = -a1r, A = -a2r.
template <int D, bool PERIODIC>
__device__ __forceinline__ cf seed_eval(const Rec<D> &r, const float *ds, const float *h, bool cont,
                                        const ProbArgs &P, cf &rr, cf &qq, int *kind = nullptr,
                                        bool skip_negligible = false) {
    float Dl[D];
    float th = r.th0;
#pragma unroll
    for (int i = 0; i < D; ++i) {
        Dl[i] = ds[i] + r.d0[i];
        if (PERIODIC && P.periodic[i]) Dl[i] -= (float)P.L[i] * rintf(Dl[i] / (float)P.L[i]);
        th = fmaf(r.wp[i], ds[i], th);
    }
    th += quad<D>(r.q, Dl);
    const float chi = quad<D>(r.p, Dl);
    cf z = cexpf_(-chi, th);
    z.re *= r.amp;
    z.im *= r.amp;
    if (cont) {
        float wh = 0.0f;
#pragma unroll
        for (int i = 0; i < D; ++i) wh = fmaf(r.wp[i], h[i], wh);
        const float a1r = -bilin2<D>(r.p, h, Dl), a1i = wh + bilin2<D>(r.q, h, Dl);
        const float a2r = -quad<D>(r.p, h), a2i = quad<D>(r.q, h);
        rr = cexpf_(a1r + a2r, a1i + a2i);
        qq = cexpf_(2.0f * a2r, 2.0f * a2i);
        if (kind) {
            const float Aq = -a2r, Bq = -a1r;
            const float kv = Aq > 0.0f ? fminf(fmaxf(-Bq / (2.0f * Aq), 0.0f), (float)(GS - 1)) : 0.0f;
            const float kl = (float)(GS - 1);
            const float chi_min = fminf(fminf(chi, chi + kl * (Bq + Aq * kl)), chi + kv * (Bq + Aq * kv));
            if (skip_negligible && chi_min > kNegligibleEfolds)
                *kind = kRunNegligible;
            else if (chi > kRecurrenceEfolds || a1r + a2r > kRecurrenceEfolds || -2.0f * a2r > kRecurrenceEfolds)
                *kind = kRunDirect;
            else
                *kind = kRunRecurrence;
        }
    }
    return z;
}

template <int D>
__device__ __forceinline__ bool survives(const Cull<D> &cb, float c0, float ta, float tb, const TileInfo<D> &ti,
                                         const ProbArgs &P, float cutoff) {
    if (!cb.ok || cutoff <= 0.0f) return true;
    float d2 = 0.0f;
#pragma unroll
    for (int i = 0; i < D; ++i) {
        if (P.periodic[i]) continue;
        const float v = c0 * cb.dir[i];
        const float xa = fmaf(v, ta, cb.x0[i]), xb = fmaf(v, tb, cb.x0[i]);
        const float mn = fminf(xa, xb), mx = fmaxf(xa, xb);
        const float gap = fmaxf(0.0f, fmaxf(ti.lo[i] - mx, mn - ti.hi[i]));
        d2 = fmaf(gap, gap, d2);
    }
    const float k = fabsf(c0) * fmaxf(fabsf(ta), fabsf(tb)) * cb.inv_np;
    const float lam = 1.0f / (1.0f / cb.bmin + k * k * cb.bmax);
    return 0.5f * cb.w * lam * d2 * 0.999f <= cutoff;
}

// ------------------------------------------------------------------ prep
// Sort key: Morton order of coarse cells (32 per axis), row-major inside a
// cell, so axis-aligned lines and planes form evenly spaced runs.
template <int D>
__global__ void sensor_key_kernel(const double *sens, int64_t ns, ProbArgs P, uint32_t *key, int32_t *val) {
    const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (s >= ns) return;
    const int bits = D == 1 ? 31 : (D == 2 ? 16 : 10);
    const int cellbits = 5;
    const int lowbits = bits - cellbits;
    uint32_t q[D];
#pragma unroll
    for (int i = 0; i < D; ++i) {
        double u = sens[s * D + i] / P.L[i];
        u = fmin(fmax(u, 0.0), 1.0 - 1e-12);
        q[i] = (uint32_t)(u * (double)(1u << bits));
    }
    uint32_t k = 0;
    if (D == 1) {
        k = q[0];
    } else {
        for (int b = cellbits - 1; b >= 0; --b)
#pragma unroll
            for (int i = 0; i < D; ++i) k = (k << 1) | ((q[i] >> (lowbits + b)) & 1u);
#pragma unroll
        for (int i = 0; i < D; ++i) k = (k << lowbits) | (q[i] & ((1u << lowbits) - 1u));
    }
    key[s] = k;
    val[s] = (int32_t)s;
}

// Per tile: anchor, bounding box, FP32 offsets, steps, run starts and the
// per-group fast flag (one straight run of GS sensors, no periodic wrap).
template <int D>
__global__ void tile_kernel(const double *sens, const int32_t *perm, const int32_t *offs, ProbArgs P,
                            TileInfo<D> *tiles, float *ds, float *hn, uint8_t *seed, uint8_t *gfast,
                            double *sorted) {
    const int64_t tile = blockIdx.x;
    const int64_t first = offs[tile];
    const int cnt = offs[tile + 1] - offs[tile];
    __shared__ double lo[D], hi[D];
    __shared__ double pos[TS][D];
    for (int k = threadIdx.x; k < cnt; k += blockDim.x)
        for (int i = 0; i < D; ++i) pos[k][i] = sens[(int64_t)perm[first + k] * D + i];
    __syncthreads();
    bool any_periodic = false;
    for (int i = 0; i < D; ++i) any_periodic |= (P.periodic[i] != 0);
    if (threadIdx.x == 0) {
        for (int i = 0; i < D; ++i) {
            double a = 1e300, b = -1e300;
            for (int k = 0; k < cnt; ++k) {
                a = fmin(a, pos[k][i]);
                b = fmax(b, pos[k][i]);
            }
            lo[i] = a;
            hi[i] = b;
            tiles[tile].s0[i] = 0.5 * (a + b);
            tiles[tile].lo[i] = (float)a;
            tiles[tile].hi[i] = (float)b;
        }
        // run starts: a run continues while the step stays the same
        bool have_h = false;
        double hh[D];
        unsigned fastmask = 0;
        for (int k = 0; k < TS; ++k) {
            bool s = true;
            if (k < cnt) {
                s = (k % GS == 0) || any_periodic;
                if (!s) {
                    double st[D], n2 = 0.0, e2 = 0.0;
                    for (int i = 0; i < D; ++i) {
                        st[i] = pos[k][i] - pos[k - 1][i];
                        n2 += st[i] * st[i];
                    }
                    if (!have_h) {
                        for (int i = 0; i < D; ++i) hh[i] = st[i];
                        have_h = n2 > 0.0;
                        s = !have_h;
                    } else {
                        for (int i = 0; i < D; ++i) e2 += (st[i] - hh[i]) * (st[i] - hh[i]);
                        s = e2 > 1e-12 * n2;
                    }
                }
                seed[first + k] = s ? 1 : 0;
            }
            if (s) have_h = false;
            if (k % GS == 0) fastmask = 1;
            if (k % GS != 0 && s) fastmask = 0;
            if (k % GS == GS - 1) gfast[tile * NW + k / GS] = (fastmask && (k < cnt) && !any_periodic) ? 1 : 0;
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < cnt; k += blockDim.x) {
        for (int i = 0; i < D; ++i) {
            const double c = 0.5 * (lo[i] + hi[i]);
            ds[(first + k) * D + i] = (float)(pos[k][i] - c);
            hn[(first + k) * D + i] = (k + 1 < cnt) ? (float)(pos[k + 1][i] - pos[k][i]) : 0.0f;
            sorted[(first + k) * D + i] = pos[k][i];
        }
    }
}

__global__ void fixed_offsets_kernel(int32_t *offs, int64_t n_tiles, int64_t ns) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i <= n_tiles) offs[i] = (int32_t)min((int64_t)i * TS, ns);
}

template <int D>
__global__ void cull_prep_kernel(BeamArgs B, Cull<D> *out) {
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= B.n) return;
    Cull<D> c;
    double n2 = 0.0;
    for (int i = 0; i < D; ++i) n2 += B.p0[j * D + i] * B.p0[j * D + i];
    const double np = sqrt(n2);
    float bmin = 1e30f, bmax = 0.0f;
    int ok = 1;
    for (int i = 0; i < D; ++i) {
        c.x0[i] = (float)B.x0[j * D + i];
        c.dir[i] = (float)(B.p0[j * D + i] / np);
        const double re = B.alpha[2 * (j * D + i)], im = B.alpha[2 * (j * D + i) + 1];
        if (re != 0.0 || !(im > 0.0)) ok = 0;
        bmin = fminf(bmin, (float)im);
        bmax = fmaxf(bmax, (float)im);
    }
    c.bmin = bmin;
    c.bmax = bmax;
    c.w = (float)B.omega[j];
    c.inv_np = (float)(1.0 / np);
    c.ok = ok && np > 0.0;
    out[j] = c;
}

// data (nt, ns) in caller order -> (ns, nt) in sorted sensor order.
__global__ void transpose_permute_kernel(const float *data, const int32_t *perm, int64_t nt, int64_t ns, float *out) {
    __shared__ float tile[32][33];
    const int64_t s0 = (int64_t)blockIdx.x * 32, t0 = (int64_t)blockIdx.y * 32;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int64_t t = t0 + k, s = s0 + threadIdx.x;
        tile[k][threadIdx.x] = (t < nt && s < ns) ? data[t * ns + perm[s]] : 0.0f;
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int64_t s = s0 + k, t = t0 + threadIdx.x;
        if (s < ns && t < nt) out[s * nt + t] = tile[threadIdx.x][k];
    }
}

// ------------------------------------------------------------------ trajectories
// Records written by msgb_rk4_trajectories (rec32) for a chunk of beams, the
// per-time-tile culling boxes, and the Kahan state carried across chunks.
template <int D>
struct TrajSrc {
    int64_t nb, b_first;
    const BeamTime<D> *rec;   // dense: (nt, nb)
    const float *cull;        // dense: (n_tt, nb, 2D + 1)
    const int32_t *slot;      // compact: (n_tt, nb) block or -1
    const BeamTime<D> *pool;  // compact: (blocks, TT)
    const float *pool_cull;   // compact: (blocks, 2D + 1)
    float *state;             // (2, nt, ns) Kahan sum / compensation, sorted sensor order
    int first, last;
};

template <int D>
__device__ __forceinline__ bool traj_survives(const TrajSrc<D> &T, int64_t bl, int64_t tt, const TileInfo<D> &ti,
                                              float cutoff) {
    const float *c;
    if (T.pool) {
        const int32_t blk = T.slot[tt * T.nb + bl];
        if (blk < 0) return false;  // no sensor tile within the cutoff: not stored
        if (cutoff <= 0.0f) return true;
        c = T.pool_cull + (int64_t)blk * (2 * D + 1);
    } else {
        if (cutoff <= 0.0f) return true;
        c = T.cull + (tt * T.nb + bl) * (2 * D + 1);
    }
    float d2 = 0.0f;
#pragma unroll
    for (int i = 0; i < D; ++i) {
        const float gap = fmaxf(0.0f, fmaxf(ti.lo[i] - c[D + i], c[i] - ti.hi[i]));
        d2 = fmaf(gap, gap, d2);
    }
    return c[2 * D] * d2 * 0.999f <= cutoff;
}

template <int D>
__device__ __forceinline__ void traj_beam_time(const BeamArgs &B, const TrajSrc<D> &T, int64_t bl, int64_t k,
                                               BeamTime<D> &bt) {
    if (T.pool)
        bt = T.pool[(int64_t)T.slot[(k / TT) * T.nb + bl] * TT + k % TT];
    else
        bt = T.rec[k * T.nb + bl];
    const int64_t b = T.b_first + bl;
    const int64_t j = b < B.n ? b : b - B.n;
    // the coefficient's amplitude and phase join the record's FP32 |A| and
    // arg A in FP32 (the record already holds them to FP32 precision)
    const float ar = (float)B.a0[2 * j], ai = (float)B.a0[2 * j + 1];
    bt.amp *= hypotf(ar, ai);
    bt.ang += atan2f(ai, (ar == 0.0f && ai == 0.0f) ? 1e-12f : ar);
}

// ------------------------------------------------------------------ forward
template <int D>
__device__ __forceinline__ void load_rec(const float (*rec)[G][TT], int gl, int lane, Rec<D> &r) {
    float *rf = reinterpret_cast<float *>(&r);
#pragma unroll
    for (int f = 0; f < Rec<D>::NF; ++f) rf[f] = rec[f][gl][lane];
}

__device__ __forceinline__ void kahan_add(float &acc, float &cmp, float v) {
    const float y = v - cmp;
    const float t = acc + y;
    cmp = (t - acc) - y;
    acc = t;
}

// Persistent CTAs take (time tile, sensor tile) work items from a counter.
// Warp w owns sensor group w (GS sensors) of the tile; lane l owns time l.
// Beams are evaluated two at a time (independent recurrence chains).
template <int D, bool PERIODIC, bool TRAJ>
__global__ void __launch_bounds__(THREADS, 2)
fwd32_kernel(ProbArgs P, BeamArgs B, const Cull<D> *cull, const TileInfo<D> *tiles, const int32_t *offs,
             const float *ds_g, const float *hn_g, const uint8_t *seed_g, const uint8_t *gfast_g,
             const int32_t *perm, float cutoff, float *out, unsigned long long *eval_count, int *work, int n_st,
             int n_tiles, TrajSrc<D> T) {
    constexpr int NF = Rec<D>::NF;
    __shared__ float rec[NF][G][TT];
    __shared__ float sds[TS][D], shn[TS][D];
    __shared__ uint8_t sseed[TS + 1];
    __shared__ int64_t surv[2 * THREADS];
    __shared__ int warp_cnt[NW];
    __shared__ int tile_s, nsurv_s;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    unsigned long long evals = 0;
    while (true) {
        if (tid == 0) tile_s = atomicAdd(work, 1);
        __syncthreads();
        const int tile = tile_s;
        if (tile >= n_tiles) break;
        const int64_t st = tile % n_st, tt = tile / n_st;
        const int64_t s_first = offs[st], t_first = tt * TT;
        const int s_cnt = offs[st + 1] - offs[st];
        const int t_cnt = (int)min((int64_t)TT, P.nt - t_first);
        const TileInfo<D> ti = tiles[st];
        const float ta = (float)P.ts[t_first], tb = (float)P.ts[t_first + t_cnt - 1];
        for (int k = tid; k < TS; k += THREADS) {
#pragma unroll
            for (int i = 0; i < D; ++i) {
                sds[k][i] = k < s_cnt ? ds_g[(s_first + k) * D + i] : 0.0f;
                shn[k][i] = k < s_cnt ? hn_g[(s_first + k) * D + i] : 0.0f;
            }
            sseed[k] = k < s_cnt ? seed_g[s_first + k] : 1;
        }
        if (tid == 0) sseed[TS] = 1;
        const bool fast = gfast_g[st * NW + warp] != 0;
        const int gbase = warp * GS;
        const bool active = gbase < s_cnt;
        // Kahan sums of sensors 2h and 2h + 1 in .x and .y
        float2 acc2[GS / 2], cmp2[GS / 2];
#pragma unroll
        for (int h = 0; h < GS / 2; ++h) acc2[h] = make_float2(0.0f, 0.0f), cmp2[h] = make_float2(0.0f, 0.0f);
        if (TRAJ && !T.first && lane < t_cnt && active) {
            const int64_t t = t_first + lane;
#pragma unroll
            for (int k = 0; k < GS; ++k) {
                const int s = gbase + k;
                if (s < s_cnt) {
                    const float a = T.state[t * P.ns + s_first + s];
                    const float c = T.state[(P.nt + t) * P.ns + s_first + s];
                    if (k & 1)
                        acc2[k / 2].y = a, cmp2[k / 2].y = c;
                    else
                        acc2[k / 2].x = a, cmp2[k / 2].x = c;
                }
            }
        }
        const int64_t nbeam = TRAJ ? T.nb : B.n;

        for (int64_t j0 = 0; j0 < nbeam; j0 += THREADS) {
            const int64_t j = j0 + tid;
            bool keep_p = false, keep_m = false;
            if (j < nbeam) {
                if (TRAJ) {
                    keep_p = traj_survives<D>(T, j, tt, ti, cutoff);
                } else {
                    const Cull<D> cb = cull[j];
                    keep_p = mode_on(B.modes, 0) && survives<D>(cb, (float)P.c, ta, tb, ti, P, cutoff);
                    keep_m = mode_on(B.modes, 1) && survives<D>(cb, -(float)P.c, ta, tb, ti, P, cutoff);
                }
            }
            const unsigned bp = __ballot_sync(0xffffffffu, keep_p);
            const unsigned bm = __ballot_sync(0xffffffffu, keep_m);
            if (lane == 0) warp_cnt[warp] = __popc(bp) + __popc(bm);
            __syncthreads();
            int off = 0, tot = 0;
#pragma unroll
            for (int w = 0; w < NW; ++w) {
                if (w < warp) off += warp_cnt[w];
                tot += warp_cnt[w];
            }
            const unsigned lt = (1u << lane) - 1u;
            if (keep_p) surv[off + __popc(bp & lt)] = j;
            if (keep_m) surv[off + __popc(bp) + __popc(bm & lt)] = j + B.n;
            if (tid == 0) nsurv_s = tot;
            __syncthreads();
            const int nsurv = nsurv_s;
            evals += (unsigned long long)nsurv * (unsigned long long)t_cnt * (unsigned long long)s_cnt;
            for (int g0 = 0; g0 < nsurv; g0 += G) {
                {
                    const int gl = tid / TT, tloc = tid % TT;
                    Rec<D> r;
                    if (g0 + gl < nsurv && tloc < t_cnt) {
                        BeamTime<D> bt;
                        if (TRAJ)
                            traj_beam_time<D>(B, T, surv[g0 + gl], t_first + tloc, bt);
                        else
                            beam_time<D>(P, B, surv[g0 + gl], P.ts[t_first + tloc], bt);
                        anchor<D>(P, bt, ti.s0, r);
                    } else {
#pragma unroll
                        for (int i = 0; i < D; ++i) r.d0[i] = 0.0f, r.wp[i] = 0.0f;
#pragma unroll
                        for (int q = 0; q < Sym<D>::S; ++q) r.q[q] = 0.0f, r.p[q] = 0.0f;
                        r.th0 = 0.0f;
                        r.amp = 0.0f;
                    }
                    const float *rf = reinterpret_cast<const float *>(&r);
#pragma unroll
                    for (int f = 0; f < NF; ++f) rec[f][gl][tloc] = rf[f];
                }
                __syncthreads();
                const int ng = min(G, nsurv - g0);
                if (active) {
                    for (int gl = 0; gl < ng; gl += 2) {
                        Rec<D> ra, rb;
                        load_rec<D>(rec, gl, lane, ra);
                        load_rec<D>(rec, gl + 1, lane, rb);  // zero-amplitude record when gl + 1 == ng
                        cf za, fa, qa, zb, fb, qb;
                        int ka = kRunRecurrence, kb = kRunRecurrence;
                        if (fast) {
                            za = seed_eval<D, false>(ra, sds[gbase], shn[gbase], true, P, fa, qa, &ka, cutoff > 0.0f);
                            zb = seed_eval<D, false>(rb, sds[gbase], shn[gbase], true, P, fb, qb, &kb, cutoff > 0.0f);
                            if (ka == kRunNegligible) za = fa = qa = cf{0.0f, 0.0f};
                            if (kb == kRunNegligible) zb = fb = qb = cf{0.0f, 0.0f};
                        }
                        if (fast && ka != kRunDirect && kb != kRunDirect) {
#if MSGB_F32X2
                            // z_{k+1} = z_k f_k, f_{k+1} = f_k q for both beams in one
                            // paired instruction stream; sensors 2h, 2h + 1 share a
                            // paired Kahan update.
                            cf2 z = pack2(za, zb), f = pack2(fa, fb);
                            const cf2 q = pack2(qa, qb);
#pragma unroll
                            for (int h = 0; h < GS / 2; ++h) {
                                if (h > 0) {
                                    z = cmul2(z, f);
                                    f = cmul2(f, q);
                                }
                                const float v0 = z.re.x + z.re.y;
                                z = cmul2(z, f);
                                f = cmul2(f, q);
                                kahan_add2(acc2[h], cmp2[h], make_float2(v0, z.re.x + z.re.y));
                            }
#else
                            float v[GS];
                            v[0] = za.re + zb.re;
#pragma unroll
                            for (int k = 1; k < GS; ++k) {
                                za = cmul(za, fa);
                                fa = cmul(fa, qa);
                                zb = cmul(zb, fb);
                                fb = cmul(fb, qb);
                                v[k] = za.re + zb.re;
                            }
#pragma unroll
                            for (int h = 0; h < GS / 2; ++h) {
                                kahan_add(acc2[h].x, cmp2[h].x, v[2 * h]);
                                kahan_add(acc2[h].y, cmp2[h].y, v[2 * h + 1]);
                            }
#endif
                        } else {
                            // Rare (broken runs, out-of-range recurrences): one copy of
                            // the direct evaluation in a loop, values staged in a small
                            // array, instead of GS inlined copies (keeps the hot loop
                            // inside the instruction cache).
                            cf dummy_r, dummy_q;
                            float v[GS];
#pragma unroll 1
                            for (int k = 0; k < GS; ++k) {
                                const int s = gbase + k;
                                const cf za = seed_eval<D, PERIODIC>(ra, sds[s], shn[s], false, P, dummy_r, dummy_q);
                                const cf zb = seed_eval<D, PERIODIC>(rb, sds[s], shn[s], false, P, dummy_r, dummy_q);
                                v[k] = za.re + zb.re;
                            }
#pragma unroll
                            for (int h = 0; h < GS / 2; ++h) {
                                kahan_add(acc2[h].x, cmp2[h].x, v[2 * h]);
                                kahan_add(acc2[h].y, cmp2[h].y, v[2 * h + 1]);
                            }
                        }
                    }
                }
                __syncthreads();
            }
        }
        if (lane < t_cnt && active) {
            const int64_t t = t_first + lane;
#pragma unroll
            for (int k = 0; k < GS; ++k) {
                const int s = gbase + k;
                if (s < s_cnt) {
                    const float a = (k & 1) ? acc2[k / 2].y : acc2[k / 2].x;
                    const float c = (k & 1) ? cmp2[k / 2].y : cmp2[k / 2].x;
                    if (TRAJ && !T.last) {
                        T.state[t * P.ns + s_first + s] = a;
                        T.state[(P.nt + t) * P.ns + s_first + s] = c;
                    } else {
                        out[t * P.ns + perm[s_first + s]] = a - c;
                    }
                }
            }
        }
        __syncthreads();
    }
    if (eval_count && tid == 0 && evals) atomicAdd(eval_count, evals);
}

// ------------------------------------------------------------------ adjoint
// Deterministic tile-parallel transpose (no floating-point atomics).
//
// Work item = (time tile tt, range of RJ consecutive beam indices j): for the
// homogeneous entry point j is a selected coefficient and both of its modes
// are summed; for trajectories j is a beam of the chunk.  Items run tt-major,
// so consecutive items read the same time tile of the data.  For each sensor
// tile in order, the CTA loads the tile's positions (shared memory) and data
// (registers: warp w holds sensor group w, lane l time l), tests the range's
// beams for survival, and for every pair of surviving beams runs the
// forward's recurrence while the lane accumulates sum_s d(t, s) conj(z(t, s)).
// The pair's partials are reduced over the 32 times (FP32 shuffles) and over
// the 8 warps (FP64), in fixed orders, into the range's per-beam FP64
// accumulators in shared memory (one owner thread per beam per pass).  The
// item then writes every accumulator (zeros included) to part[tt][slot], and
// reduce_parts_kernel sums part over the time tiles in order.  Each partial
// has one writer and every sum has a fixed order, so the result is
// bit-identical between runs; the work counter only hands out items.
constexpr int NACC = 2048;  // accumulator slots (re, im FP64) per item

template <bool TRAJ>
struct AdjRange {
    static constexpr int RJ = TRAJ ? NACC : NACC / 2;  // beam indices per item
};

template <int D, bool PERIODIC, bool TRAJ>
__global__ void __launch_bounds__(THREADS, 2)
adj32_kernel(ProbArgs P, BeamArgs B, const Cull<D> *cull, const TileInfo<D> *tiles, const int32_t *offs,
             const float *ds_g, const float *hn_g, const uint8_t *gfast_g, const float *dataT, float cutoff,
             double *part, unsigned long long *eval_count, int *work, int n_st, int n_ranges, int n_items,
             TrajSrc<D> T) {
    constexpr int NF = Rec<D>::NF;
    constexpr int RJ = AdjRange<TRAJ>::RJ;
    __shared__ float rec[NF][G][TT];
    __shared__ float sds[TS][D], shn[TS][D];
    __shared__ int32_t surv[2 * THREADS];
    __shared__ int warp_cnt[NW];
    __shared__ double wpart[NW][G][2];
    __shared__ int item_s, nsurv_s;
    extern __shared__ double acc_smem[];  // (NACC, 2)

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int64_t nbeam = TRAJ ? T.nb : B.n;
    const int64_t nslots = TRAJ ? T.nb : 2 * B.n;
    unsigned long long evals = 0;
    for (int q = tid; q < 2 * NACC; q += THREADS) acc_smem[q] = 0.0;
    while (true) {
        if (tid == 0) item_s = atomicAdd(work, 1);
        __syncthreads();
        const int item = item_s;
        if (item >= n_items) break;
        const int64_t tt = item / n_ranges, r0 = (int64_t)(item % n_ranges) * RJ;
        const int64_t r1 = min(r0 + RJ, nbeam);
        const int64_t t_first = tt * TT;
        const int t_cnt = (int)min((int64_t)TT, P.nt - t_first);
        const float ta = (float)P.ts[t_first], tb = (float)P.ts[t_first + t_cnt - 1];
        const bool tv = lane < t_cnt;
        for (int st = 0; st < n_st; ++st) {
            const int64_t s_first = offs[st];
            const int s_cnt = offs[st + 1] - offs[st];
            if (s_cnt <= 0) continue;
            const TileInfo<D> ti = tiles[st];
            __syncthreads();  // the previous tile's passes are done with sds / shn
            for (int k = tid; k < TS; k += THREADS) {
#pragma unroll
                for (int i = 0; i < D; ++i) {
                    sds[k][i] = k < s_cnt ? ds_g[(s_first + k) * D + i] : 0.0f;
                    shn[k][i] = k < s_cnt ? hn_g[(s_first + k) * D + i] : 0.0f;
                }
            }
            const bool fast = gfast_g[st * NW + warp] != 0;
            const int gbase = warp * GS;
            const bool active = gbase < s_cnt;
            const float *dcol = dataT + (int64_t)s_first * P.nt + t_first + lane;
            float dv[GS];
#pragma unroll
            for (int k = 0; k < GS; ++k)
                dv[k] = (tv && gbase + k < s_cnt) ? __ldg(dcol + (int64_t)(gbase + k) * P.nt) : 0.0f;

            for (int64_t j0 = r0; j0 < r1; j0 += THREADS) {
                const int64_t j = j0 + tid;
                bool keep_p = false, keep_m = false;
                if (j < r1) {
                    if (TRAJ) {
                        keep_p = traj_survives<D>(T, j, tt, ti, cutoff);
                    } else {
                        const Cull<D> cb = cull[j];
                        keep_p = mode_on(B.modes, 0) && survives<D>(cb, (float)P.c, ta, tb, ti, P, cutoff);
                        keep_m = mode_on(B.modes, 1) && survives<D>(cb, -(float)P.c, ta, tb, ti, P, cutoff);
                    }
                }
                const unsigned bp = __ballot_sync(0xffffffffu, keep_p);
                const unsigned bm = __ballot_sync(0xffffffffu, keep_m);
                if (lane == 0) warp_cnt[warp] = __popc(bp) + __popc(bm);
                __syncthreads();  // also: sds / shn loaded
                int off = 0, tot = 0;
#pragma unroll
                for (int w = 0; w < NW; ++w) {
                    if (w < warp) off += warp_cnt[w];
                    tot += warp_cnt[w];
                }
                // local slot: beam j - r0 (mode +1 / trajectories), RJ + j - r0 (mode -1)
                const unsigned lt = (1u << lane) - 1u;
                if (keep_p) surv[off + __popc(bp & lt)] = (int32_t)(j - r0);
                if (keep_m) surv[off + __popc(bp) + __popc(bm & lt)] = (int32_t)(RJ + j - r0);
                if (tid == 0) nsurv_s = tot;
                __syncthreads();
                const int nsurv = nsurv_s;
                evals += (unsigned long long)nsurv * (unsigned long long)t_cnt * (unsigned long long)s_cnt;
                for (int g0 = 0; g0 < nsurv; g0 += G) {
                    {
                        const int gl = tid / TT, tloc = tid % TT;
                        Rec<D> r;
                        if (g0 + gl < nsurv && tloc < t_cnt) {
                            const int q = surv[g0 + gl];
                            const int64_t b = TRAJ ? r0 + q : (q < RJ ? r0 + q : B.n + r0 + q - RJ);
                            BeamTime<D> bt;
                            if (TRAJ)
                                traj_beam_time<D>(B, T, b, t_first + tloc, bt);
                            else
                                beam_time<D>(P, B, b, P.ts[t_first + tloc], bt);
                            anchor<D>(P, bt, ti.s0, r);
                        } else {
#pragma unroll
                            for (int i = 0; i < D; ++i) r.d0[i] = 0.0f, r.wp[i] = 0.0f;
#pragma unroll
                            for (int q = 0; q < Sym<D>::S; ++q) r.q[q] = 0.0f, r.p[q] = 0.0f;
                            r.th0 = 0.0f;
                            r.amp = 0.0f;
                        }
                        const float *rf = reinterpret_cast<const float *>(&r);
#pragma unroll
                        for (int f = 0; f < NF; ++f) rec[f][gl][tloc] = rf[f];
                    }
                    __syncthreads();
                    const int ng = min(G, nsurv - g0);
                    for (int gl = 0; gl < ng; gl += 2) {
                        float2 ar = make_float2(0.0f, 0.0f), ai = make_float2(0.0f, 0.0f);
                        if (active) {
                            Rec<D> ra, rb;
                            load_rec<D>(rec, gl, lane, ra);
                            load_rec<D>(rec, gl + 1, lane, rb);  // zero-amplitude record when gl + 1 == ng
                            cf za, fa, qa, zb, fb, qb;
                            int ka = kRunRecurrence, kb = kRunRecurrence;
                            if (fast) {
                                za = seed_eval<D, false>(ra, sds[gbase], shn[gbase], true, P, fa, qa, &ka, cutoff > 0.0f);
                                zb = seed_eval<D, false>(rb, sds[gbase], shn[gbase], true, P, fb, qb, &kb, cutoff > 0.0f);
                                if (ka == kRunNegligible) za = fa = qa = cf{0.0f, 0.0f};
                                if (kb == kRunNegligible) zb = fb = qb = cf{0.0f, 0.0f};
                            }
                            if (fast && ka != kRunDirect && kb != kRunDirect) {
#if MSGB_F32X2
                                cf2 z = pack2(za, zb), f = pack2(fa, fb);
                                const cf2 q = pack2(qa, qb);
#pragma unroll
                                for (int k = 0; k < GS; ++k) {
                                    if (k > 0) {
                                        z = cmul2(z, f);
                                        f = cmul2(f, q);
                                    }
                                    const float2 dk = make_float2(dv[k], dv[k]);
                                    ar = __ffma2_rn(dk, z.re, ar);
                                    ai = __ffma2_rn(neg2(dk), z.im, ai);
                                }
#else
#pragma unroll
                                for (int k = 0; k < GS; ++k) {
                                    if (k > 0) {
                                        za = cmul(za, fa);
                                        fa = cmul(fa, qa);
                                        zb = cmul(zb, fb);
                                        fb = cmul(fb, qb);
                                    }
                                    ar.x = fmaf(dv[k], za.re, ar.x);
                                    ai.x = fmaf(-dv[k], za.im, ai.x);
                                    ar.y = fmaf(dv[k], zb.re, ar.y);
                                    ai.y = fmaf(-dv[k], zb.im, ai.y);
                                }
#endif
                            } else {
                                // rare: broken runs, out-of-range recurrences
                                cf dummy_r, dummy_q;
#pragma unroll 1
                                for (int k = 0; k < GS; ++k) {
                                    const int s = gbase + k;
                                    const float d = (tv && s < s_cnt) ? __ldg(dcol + (int64_t)s * P.nt) : 0.0f;
                                    const cf za = seed_eval<D, PERIODIC>(ra, sds[s], shn[s], false, P, dummy_r, dummy_q);
                                    const cf zb = seed_eval<D, PERIODIC>(rb, sds[s], shn[s], false, P, dummy_r, dummy_q);
                                    ar.x = fmaf(d, za.re, ar.x);
                                    ai.x = fmaf(-d, za.im, ai.x);
                                    ar.y = fmaf(d, zb.re, ar.y);
                                    ai.y = fmaf(-d, zb.im, ai.y);
                                }
                            }
                        }
                        // over the 32 times (the partials are sums of 16 terms): a
                        // reduce-scatter of the pair's four partials, 6 shuffles
                        // instead of 20.  Lanes 0, 8, 16, 24 end with the sums of
                        // ar.x, ar.y, ai.x, ai.y; FP64 from here on.
                        {
                            const bool u4 = (lane & 16) != 0, u3 = (lane & 8) != 0;
                            float k0 = u4 ? ai.x : ar.x, k1 = u4 ? ai.y : ar.y;
                            k0 += __shfl_xor_sync(0xffffffffu, u4 ? ar.x : ai.x, 16);
                            k1 += __shfl_xor_sync(0xffffffffu, u4 ? ar.y : ai.y, 16);
                            float v = u3 ? k1 : k0;
                            v += __shfl_xor_sync(0xffffffffu, u3 ? k0 : k1, 8);
                            v += __shfl_xor_sync(0xffffffffu, v, 4);
                            v += __shfl_xor_sync(0xffffffffu, v, 2);
                            v += __shfl_xor_sync(0xffffffffu, v, 1);
                            // beam gl + u3 (gl + 1 < G: gl is even and G is even), re / im by u4
                            if ((lane & 7) == 0) wpart[warp][gl + (u3 ? 1 : 0)][u4 ? 1 : 0] = (double)v;
                        }
                    }
                    __syncthreads();
                    if (tid < ng) {
                        double re = 0.0, im = 0.0;
#pragma unroll
                        for (int w = 0; w < NW; ++w) {
                            re += wpart[w][tid][0];
                            im += wpart[w][tid][1];
                        }
                        const int q = surv[g0 + tid];  // distinct within a pass: one owner per slot
                        acc_smem[2 * q] += re;
                        acc_smem[2 * q + 1] += im;
                    }
                }
            }
        }
        __syncthreads();
        // every slot of the item, zeros included, then clear for the next item
        for (int q = tid; q < NACC; q += THREADS) {
            const int64_t jl = TRAJ ? q : (q < RJ ? q : q - RJ);
            const int64_t j = r0 + jl;
            if (j < r1) {
                const int64_t slot = TRAJ ? j : (q < RJ ? j : B.n + j);
                double *dst = part + 2 * (tt * nslots + slot);
                dst[0] = acc_smem[2 * q];
                dst[1] = acc_smem[2 * q + 1];
            }
            acc_smem[2 * q] = 0.0;
            acc_smem[2 * q + 1] = 0.0;
        }
    }
    if (eval_count && tid == 0 && evals) atomicAdd(eval_count, evals);
}

// g[j] = sum over time tiles, in order, of part[tt][j] (trajectories) or of
// part[tt][j] + part[tt][n + j] (both modes of coefficient j).
__global__ void reduce_parts_kernel(const double *part, int64_t n_tt, int64_t nslots, int64_t n_out, int both_modes,
                                    double *g) {
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= n_out) return;
    double re = 0.0, im = 0.0;
    for (int64_t tt = 0; tt < n_tt; ++tt) {
        const double *p = part + 2 * (tt * nslots + j);
        re += p[0];
        im += p[1];
        if (both_modes) {
            re += p[2 * n_out];
            im += p[2 * n_out + 1];
        }
    }
    g[2 * j] = re;
    g[2 * j + 1] = im;
}

// ------------------------------------------------------------------ workspace
struct Layout {
    size_t keys_in, keys_out, vals_in, vals_out, cub, tiles, offs, gfast, ds, hn, seed, sorted, cull, data, work, part,
        total;
    size_t cub_bytes;
    int64_t n_st;
    int64_t cull_cap;  // beams the culling table has room for
};

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

int64_t tile_count(const msgb_problem *p, const msgb_sum_opts *o) {
    if (o && o->tiling) return o->tiling->n_tiles;
    return (p->ns + TS - 1) / TS;
}

Layout layout(const msgb_problem *p, int64_t n_beams, bool with_data, int64_t n_st) {
    Layout l{};
    const int D = p->ndim;
    const int64_t ns = p->ns;
    l.n_st = n_st;
    size_t cub_bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, cub_bytes, (const uint32_t *)nullptr, (uint32_t *)nullptr,
                                    (const int32_t *)nullptr, (int32_t *)nullptr, (int)ns);
    l.cub_bytes = cub_bytes;
    size_t o = 0;
    l.keys_in = o; o = align256(o + ns * 4);
    l.keys_out = o; o = align256(o + ns * 4);
    l.vals_in = o; o = align256(o + ns * 4);
    l.vals_out = o; o = align256(o + ns * 4);
    l.cub = o; o = align256(o + cub_bytes);
    l.tiles = o; o = align256(o + n_st * sizeof(TileInfo<3>));
    l.offs = o; o = align256(o + (n_st + 1) * 4);
    l.gfast = o; o = align256(o + n_st * NW);
    l.ds = o; o = align256(o + ns * D * 4);
    l.hn = o; o = align256(o + ns * D * 4);
    l.seed = o; o = align256(o + ns + 1);
    l.sorted = o; o = align256(o + ns * D * 8);
    l.cull_cap = n_beams > 0 ? n_beams : 1;
    l.cull = o; o = align256(o + l.cull_cap * sizeof(Cull<3>));
    l.data = o; o = align256(o + (with_data ? p->nt * ns * 4 : 0));
    l.work = o; o = align256(o + 64);
    // adjoint partials: one complex FP64 per (time tile, beam mode) of the coefficients
    l.part = o; o = align256(o + (with_data ? (size_t)((p->nt + TT - 1) / TT) * 2 * (n_beams > 0 ? n_beams : 0) * 16 : 0));
    l.total = o;
    return l;
}

// Adjoint partials of a trajectory chunk of nb beams: (n_tt, nb) complex FP64.
size_t traj_part_bytes(const msgb_problem *p, int64_t nb) {
    return align256((size_t)((p->nt + TT - 1) / TT) * (size_t)(nb > 0 ? nb : 0) * 16);
}

__global__ void copy_i32_kernel(const int32_t *in, int64_t n, int32_t *out) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) out[i] = in[i];
}

// Caller-provided tile offsets are clamped so that every tile lies in
// [0, ns) and holds at most TS sensors; order entries outside [0, ns) are
// replaced by 0.  (A malformed tiling gives wrong numbers, never an
// out-of-bounds access.)
__global__ void sanitize_tiling_kernel(const int32_t *offs_in, int64_t n_st, int64_t ns, int32_t *offs,
                                       int32_t *order) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i <= n_st) {
        int64_t v = offs_in[i];
        v = v < 0 ? 0 : (v > ns ? ns : v);
        offs[i] = (int32_t)v;
    }
    for (int64_t k = i; k < ns; k += (int64_t)gridDim.x * blockDim.x)
        if (order[k] < 0 || order[k] >= ns) order[k] = 0;
}

__global__ void clamp_tiles_kernel(int32_t *offs, int64_t n_st) {
    // serial pass (n_st is small): non-decreasing, at most TS per tile
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    for (int64_t i = 1; i <= n_st; ++i) {
        int32_t lo = offs[i - 1];
        int32_t v = offs[i] < lo ? lo : offs[i];
        if (v - lo > TS) v = lo + TS;
        offs[i] = v;
    }
}

template <int D>
int prep(const msgb_problem *p, const msgb_beam_set *b, const msgb_sum_opts *o, const Layout &l, char *ws,
         cudaStream_t st) {
    const int64_t ns = p->ns;
    if (b->n > l.cull_cap) return fail(MSGB_ERR_WORKSPACE, "culling table sized for %lld beams, got %lld",
                                       (long long)l.cull_cap, (long long)b->n);
    uint32_t *kin = (uint32_t *)(ws + l.keys_in), *kout = (uint32_t *)(ws + l.keys_out);
    int32_t *vin = (int32_t *)(ws + l.vals_in), *vout = (int32_t *)(ws + l.vals_out);
    int32_t *offs = (int32_t *)(ws + l.offs);
    const int blk = 256;
    if (o && o->tiling) {
        if (!o->tiling->order || !o->tiling->tile_offsets || o->tiling->n_tiles <= 0)
            return fail(MSGB_ERR_ARG, "sensor tiling: NULL arrays or no tiles");
        copy_i32_kernel<<<(unsigned)((ns + blk - 1) / blk), blk, 0, st>>>(o->tiling->order, ns, vout);
        sanitize_tiling_kernel<<<(unsigned)((l.n_st + 1 + blk - 1) / blk), blk, 0, st>>>(o->tiling->tile_offsets,
                                                                                        l.n_st, ns, offs, vout);
        clamp_tiles_kernel<<<1, 1, 0, st>>>(offs, l.n_st);
    } else {
        sensor_key_kernel<D><<<(unsigned)((ns + blk - 1) / blk), blk, 0, st>>>(p->sensors, ns, to_args(p), kin, vin);
        size_t cb = l.cub_bytes;
        cudaError_t e = cub::DeviceRadixSort::SortPairs(ws + l.cub, cb, kin, kout, vin, vout, (int)ns, 0, 32, st);
        if (e != cudaSuccess) return fail(MSGB_ERR_CUDA, "sensor sort: %s", cudaGetErrorString(e));
        fixed_offsets_kernel<<<(unsigned)((l.n_st + 1 + blk - 1) / blk), blk, 0, st>>>(offs, l.n_st, ns);
    }
    tile_kernel<D><<<(unsigned)l.n_st, 128, 0, st>>>(p->sensors, vout, offs, to_args(p), (TileInfo<D> *)(ws + l.tiles),
                                                    (float *)(ws + l.ds), (float *)(ws + l.hn), (uint8_t *)(ws + l.seed),
                                                    (uint8_t *)(ws + l.gfast), (double *)(ws + l.sorted));
    if (b->n > 0)
        cull_prep_kernel<D><<<(unsigned)((b->n + blk - 1) / blk), blk, 0, st>>>(to_args(b), (Cull<D> *)(ws + l.cull));
    return check_launch("msgb sum f32 prep");
}

int sm_count() {
    int dev = 0, n = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n;
}

template <int D, bool TRAJ>
int run_fwd(const msgb_problem *p, const msgb_beam_set *b, const msgb_sum_opts *o, char *ws, const Layout &l,
            float *out, cudaStream_t st, TrajSrc<D> T) {
    // trajectory sums cull with the records' own boxes: the closed-form
    // culling table (sized for no beams in their layout) is not built
    msgb_beam_set none{};
    if (int e = prep<D>(p, TRAJ ? &none : b, o, l, ws, st)) return e;
    const int64_t n_st = l.n_st, n_tt = (p->nt + TT - 1) / TT;
    if (n_st * n_tt > 0x7fffffffLL) return fail(MSGB_ERR_UNSUPPORTED, "msgb_sum_fwd_f32: too many tiles");
    ProbArgs P = to_args(p);
    P.sensors = (const double *)(ws + l.sorted);
    int *work = (int *)(ws + l.work);
    cudaMemsetAsync(work, 0, sizeof(int), st);
    bool periodic = false;
    for (int i = 0; i < D; ++i) periodic |= (p->periodic[i] != 0);
    const int n_tiles = (int)(n_st * n_tt);
    const int64_t want = 2LL * sm_count();
    const unsigned grid = (unsigned)(want < n_tiles ? want : n_tiles);
    auto args = [&](auto kern) {
        kern<<<grid, THREADS, 0, st>>>(P, to_args(b), (const Cull<D> *)(ws + l.cull), (const TileInfo<D> *)(ws + l.tiles),
                                       (const int32_t *)(ws + l.offs), (const float *)(ws + l.ds),
                                       (const float *)(ws + l.hn), (const uint8_t *)(ws + l.seed),
                                       (const uint8_t *)(ws + l.gfast), (const int32_t *)(ws + l.vals_out),
                                       o ? (float)o->cutoff : 0.0f, out, o ? o->eval_count : nullptr, work,
                                       (int)n_st, n_tiles, T);
    };
    if (periodic)
        args(fwd32_kernel<D, true, TRAJ>);
    else
        args(fwd32_kernel<D, false, TRAJ>);
    return check_launch("msgb_sum_fwd_f32");
}

template <int D, bool TRAJ>
int run_adj(const msgb_problem *p, const msgb_beam_set *b, const msgb_sum_opts *o, char *ws, const Layout &l,
            const float *data, double *part, double *g, cudaStream_t st, TrajSrc<D> T) {
    msgb_beam_set none{};
    if (int e = prep<D>(p, TRAJ ? &none : b, o, l, ws, st)) return e;
    dim3 tg((unsigned)((p->ns + 31) / 32), (unsigned)((p->nt + 31) / 32));
    if (tg.y > 65535u) return fail(MSGB_ERR_UNSUPPORTED, "msgb_adj_gather_f32: nt too large");
    transpose_permute_kernel<<<tg, dim3(32, 8), 0, st>>>(data, (const int32_t *)(ws + l.vals_out), p->nt, p->ns,
                                                         (float *)(ws + l.data));
    ProbArgs P = to_args(p);
    P.sensors = (const double *)(ws + l.sorted);
    bool periodic = false;
    for (int i = 0; i < D; ++i) periodic |= (p->periodic[i] != 0);
    const int64_t nw = TRAJ ? T.nb : b->n;  // beam indices j of the items
    const int64_t n_st = l.n_st, n_tt = (p->nt + TT - 1) / TT;
    const int64_t n_ranges = (nw + AdjRange<TRAJ>::RJ - 1) / AdjRange<TRAJ>::RJ;
    if (n_ranges * n_tt > 0x7fffffffLL || n_st > 0x7fffffffLL)
        return fail(MSGB_ERR_UNSUPPORTED, "msgb_adj_gather_f32: too many work items");
    int *work = (int *)(ws + l.work);
    cudaMemsetAsync(work, 0, sizeof(int), st);
    const int n_items = (int)(n_ranges * n_tt);
    const int64_t want = 2LL * sm_count();
    const unsigned grid = (unsigned)(want < n_items ? want : n_items);
    const size_t smem = (size_t)NACC * 2 * sizeof(double);
    auto args = [&](auto kern) {
        // static + dynamic shared memory exceed the default 48 KB: opt in
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        kern<<<grid, THREADS, smem, st>>>(P, to_args(b), (const Cull<D> *)(ws + l.cull),
                                          (const TileInfo<D> *)(ws + l.tiles), (const int32_t *)(ws + l.offs),
                                          (const float *)(ws + l.ds), (const float *)(ws + l.hn),
                                          (const uint8_t *)(ws + l.gfast), (const float *)(ws + l.data),
                                          o ? (float)o->cutoff : 0.0f, part, o ? o->eval_count : nullptr, work,
                                          (int)n_st, (int)n_ranges, n_items, T);
    };
    if (periodic)
        args(adj32_kernel<D, true, TRAJ>);
    else
        args(adj32_kernel<D, false, TRAJ>);
    if (int e = check_launch("msgb_adj_gather_f32")) return e;
    const int blk = 256;
    reduce_parts_kernel<<<(unsigned)((nw + blk - 1) / blk), blk, 0, st>>>(part, n_tt, TRAJ ? nw : 2 * nw, nw,
                                                                          TRAJ ? 0 : 1, g);
    return check_launch("msgb_adj_gather_f32 reduce");
}

template <int D>
TrajSrc<D> traj_src(const msgb_trajectories *t, float *state, int first, int last) {
    TrajSrc<D> T{};
    if (t) {
        T.nb = t->nb;
        T.b_first = t->b_first;
        T.rec = (const BeamTime<D> *)t->rec32;
        T.cull = t->cull;
        if (t->pool) {
            T.slot = t->slot;
            T.pool = (const BeamTime<D> *)t->pool;
            T.pool_cull = t->pool_cull;
        }
    }
    T.state = state;
    T.first = first;
    T.last = last;
    return T;
}

}  // namespace
}  // namespace msgb

using namespace msgb;

extern "C" size_t msgb_sum_f32_workspace_size(const msgb_problem *prob, int64_t n) {
    if (validate_problem(prob) || n < 0) return 0;
    // The default tiling has the most tiles a valid tiling of ns sensors needs
    // when every tile is full; reserve for one tile per 16 sensors so that
    // caller tilings with partial tiles fit as well.
    return layout(prob, n, true, (prob->ns + GS - 1) / GS).total;
}

static int check_ws(const msgb_problem *p, const msgb_beam_set *b, const msgb_sum_opts *o, bool with_data, void *ws,
                    size_t bytes, Layout &l) {
    l = layout(p, b->n, with_data, tile_count(p, o));
    if (l.n_st <= 0) return fail(MSGB_ERR_ARG, "sensor tiling has no tiles");
    if (b->n > (int64_t(1) << 26)) return fail(MSGB_ERR_UNSUPPORTED, "at most 2^26 selected coefficients");
    if (!ws || bytes < l.total)
        return fail(MSGB_ERR_WORKSPACE, "workspace too small: need %zu bytes, got %zu", l.total, bytes);
    if (((uintptr_t)ws & 255) != 0) return fail(MSGB_ERR_WORKSPACE, "workspace must be 256-byte aligned");
    if (p->ns > 0x7fffffffLL) return fail(MSGB_ERR_UNSUPPORTED, "too many sensors");
    return MSGB_OK;
}

extern "C" int msgb_sum_fwd_f32(const msgb_problem *prob, const msgb_beam_set *beams, const msgb_sum_opts *opts,
                                void *workspace, size_t workspace_bytes, float *out, msgb_stream_t stream) {
    if (int e = validate_problem(prob)) return e;
    if (int e = validate_beams(prob, beams)) return e;
    if (!out) return fail(MSGB_ERR_ARG, "msgb_sum_fwd_f32: out is NULL");
    if (prob->nt == 0 || prob->ns == 0) return MSGB_OK;
    Layout l;
    if (int e = check_ws(prob, beams, opts, false, workspace, workspace_bytes, l)) return e;
    cudaStream_t st = as_stream(stream);
    char *ws = (char *)workspace;
    switch (prob->ndim) {
        case 1: return run_fwd<1, false>(prob, beams, opts, ws, l, out, st, traj_src<1>(nullptr, nullptr, 1, 1));
        case 2: return run_fwd<2, false>(prob, beams, opts, ws, l, out, st, traj_src<2>(nullptr, nullptr, 1, 1));
        default: return run_fwd<3, false>(prob, beams, opts, ws, l, out, st, traj_src<3>(nullptr, nullptr, 1, 1));
    }
}

extern "C" int msgb_adj_gather_f32(const msgb_problem *prob, const msgb_beam_set *beams, const msgb_sum_opts *opts,
                                   void *workspace, size_t workspace_bytes, const float *data, double *g,
                                   msgb_stream_t stream) {
    if (int e = validate_problem(prob)) return e;
    if (int e = validate_beams(prob, beams)) return e;
    if (!data || !g) return fail(MSGB_ERR_ARG, "msgb_adj_gather_f32: NULL data or g");
    if (beams->n == 0) return MSGB_OK;
    if (prob->nt == 0 || prob->ns == 0) {
        cudaMemsetAsync(g, 0, sizeof(double) * 2 * beams->n, as_stream(stream));
        return check_launch("msgb_adj_gather_f32");
    }
    Layout l;
    if (int e = check_ws(prob, beams, opts, true, workspace, workspace_bytes, l)) return e;
    cudaStream_t st = as_stream(stream);
    char *ws = (char *)workspace;
    switch (prob->ndim) {
        case 1: return run_adj<1, false>(prob, beams, opts, ws, l, data, (double *)(ws + l.part), g, st,
                                         traj_src<1>(nullptr, nullptr, 1, 1));
        case 2: return run_adj<2, false>(prob, beams, opts, ws, l, data, (double *)(ws + l.part), g, st,
                                         traj_src<2>(nullptr, nullptr, 1, 1));
        default: return run_adj<3, false>(prob, beams, opts, ws, l, data, (double *)(ws + l.part), g, st,
                                          traj_src<3>(nullptr, nullptr, 1, 1));
    }
}

// ---- trajectory entry points ------------------------------------------------
static size_t traj_state_offset(const Layout &l) { return l.total; }

static size_t traj_state_bytes(const msgb_problem *p) { return align256((size_t)2 * p->nt * p->ns * sizeof(float)); }

extern "C" size_t msgb_sum_f32_traj_workspace_size(const msgb_problem *prob, int64_t nb_max) {
    if (validate_problem(prob) || nb_max < 0) return 0;
    const Layout l = layout(prob, 0, true, (prob->ns + GS - 1) / GS);
    return l.total + traj_state_bytes(prob) + traj_part_bytes(prob, nb_max);
}

// with_part: the adjoint's partials (n_tt, nb) follow the Kahan state.
static int check_traj32(const msgb_problem *p, const msgb_beam_set *b, const msgb_trajectories *t,
                        const msgb_sum_opts *o, void *ws, size_t bytes, bool with_part, Layout &l) {
    if (!t || (!t->rec32 && !t->pool)) return fail(MSGB_ERR_ARG, "FP32 trajectory records are NULL");
    if (t->pool) {
        if (!t->slot || !t->pool_cull) return fail(MSGB_ERR_ARG, "compact trajectories: slot or pool_cull is NULL");
    } else if (!t->cull && o && o->cutoff > 0.0) {
        return fail(MSGB_ERR_ARG, "culling boxes are NULL");
    }
    if (t->nb < 0 || t->b_first < 0 || t->b_first + t->nb > 2 * b->n)
        return fail(MSGB_ERR_ARG, "trajectory beam range outside [0, 2n)");
    l = layout(p, 0, true, tile_count(p, o));
    if (l.n_st <= 0) return fail(MSGB_ERR_ARG, "sensor tiling has no tiles");
    const size_t need = l.total + traj_state_bytes(p) + (with_part ? traj_part_bytes(p, t->nb) : 0);
    if (!ws || bytes < need) return fail(MSGB_ERR_WORKSPACE, "workspace too small: need %zu bytes, got %zu", need, bytes);
    if (((uintptr_t)ws & 255) != 0) return fail(MSGB_ERR_WORKSPACE, "workspace must be 256-byte aligned");
    return MSGB_OK;
}

extern "C" int msgb_sum_fwd_f32_traj(const msgb_problem *prob, const msgb_beam_set *beams,
                                     const msgb_trajectories *traj, const msgb_sum_opts *opts, int first_chunk,
                                     int last_chunk, void *workspace, size_t workspace_bytes, float *out,
                                     msgb_stream_t stream) {
    if (int e = validate_problem(prob)) return e;
    if (int e = validate_beams(prob, beams)) return e;
    if (!out) return fail(MSGB_ERR_ARG, "msgb_sum_fwd_f32_traj: out is NULL");
    if (prob->nt == 0 || prob->ns == 0) return MSGB_OK;
    Layout l;
    if (int e = check_traj32(prob, beams, traj, opts, workspace, workspace_bytes, false, l)) return e;
    cudaStream_t st = as_stream(stream);
    char *ws = (char *)workspace;
    float *state = (float *)(ws + traj_state_offset(l));
    const int f = first_chunk != 0, la = last_chunk != 0;
    switch (prob->ndim) {
        case 1: return run_fwd<1, true>(prob, beams, opts, ws, l, out, st, traj_src<1>(traj, state, f, la));
        case 2: return run_fwd<2, true>(prob, beams, opts, ws, l, out, st, traj_src<2>(traj, state, f, la));
        default: return run_fwd<3, true>(prob, beams, opts, ws, l, out, st, traj_src<3>(traj, state, f, la));
    }
}

extern "C" int msgb_adj_gather_f32_traj(const msgb_problem *prob, const msgb_beam_set *beams,
                                        const msgb_trajectories *traj, const msgb_sum_opts *opts, void *workspace,
                                        size_t workspace_bytes, const float *data, double *g, msgb_stream_t stream) {
    if (int e = validate_problem(prob)) return e;
    if (int e = validate_beams(prob, beams)) return e;
    if (!data || !g) return fail(MSGB_ERR_ARG, "msgb_adj_gather_f32_traj: NULL data or g");
    if (!traj || traj->nb == 0) return MSGB_OK;
    if (prob->nt == 0 || prob->ns == 0) {
        cudaMemsetAsync(g, 0, sizeof(double) * 2 * traj->nb, as_stream(stream));
        return check_launch("msgb_adj_gather_f32_traj");
    }
    Layout l;
    if (int e = check_traj32(prob, beams, traj, opts, workspace, workspace_bytes, true, l)) return e;
    cudaStream_t st = as_stream(stream);
    char *ws = (char *)workspace;
    double *part = (double *)(ws + traj_state_offset(l) + traj_state_bytes(prob));
    switch (prob->ndim) {
        case 1: return run_adj<1, true>(prob, beams, opts, ws, l, data, part, g, st, traj_src<1>(traj, nullptr, 1, 1));
        case 2: return run_adj<2, true>(prob, beams, opts, ws, l, data, part, g, st, traj_src<2>(traj, nullptr, 1, 1));
        default: return run_adj<3, true>(prob, beams, opts, ws, l, data, part, g, st, traj_src<3>(traj, nullptr, 1, 1));
    }
}

// ---- sensor-tile boxes (for the compact trajectory store) -------------------
namespace msgb {
namespace {
template <int D>
__global__ void tile_boxes_kernel(const TileInfo<D> *tiles, int64_t n_st, float *boxes) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n_st) return;
#pragma unroll
    for (int a = 0; a < D; ++a) {
        boxes[i * 2 * D + a] = tiles[i].lo[a];
        boxes[i * 2 * D + D + a] = tiles[i].hi[a];
    }
}

template <int D>
int tile_boxes(const msgb_problem *p, const msgb_sum_opts *o, char *ws, const Layout &l, float *boxes,
               cudaStream_t st) {
    msgb_beam_set none{};
    if (int e = prep<D>(p, &none, o, l, ws, st)) return e;
    tile_boxes_kernel<D><<<(unsigned)((l.n_st + 127) / 128), 128, 0, st>>>((const TileInfo<D> *)(ws + l.tiles),
                                                                           l.n_st, boxes);
    return check_launch("msgb_sum_f32_tile_boxes");
}
}  // namespace
}  // namespace msgb

extern "C" int64_t msgb_sum_f32_tile_count(const msgb_problem *prob, const msgb_sum_opts *opts) {
    if (validate_problem(prob)) return -1;
    return tile_count(prob, opts);
}

extern "C" int msgb_sum_f32_tile_boxes(const msgb_problem *prob, const msgb_sum_opts *opts, void *workspace,
                                       size_t workspace_bytes, float *boxes, msgb_stream_t stream) {
    if (int e = validate_problem(prob)) return e;
    if (!boxes) return fail(MSGB_ERR_ARG, "msgb_sum_f32_tile_boxes: boxes is NULL");
    if (prob->ns == 0) return MSGB_OK;
    const Layout l = layout(prob, 0, true, tile_count(prob, opts));
    if (l.n_st <= 0) return fail(MSGB_ERR_ARG, "sensor tiling has no tiles");
    if (!workspace || workspace_bytes < l.total)
        return fail(MSGB_ERR_WORKSPACE, "workspace too small: need %zu bytes, got %zu", l.total, workspace_bytes);
    if (((uintptr_t)workspace & 255) != 0) return fail(MSGB_ERR_WORKSPACE, "workspace must be 256-byte aligned");
    cudaStream_t st = as_stream(stream);
    char *ws = (char *)workspace;
    switch (prob->ndim) {
        case 1: return tile_boxes<1>(prob, opts, ws, l, boxes, st);
        case 2: return tile_boxes<2>(prob, opts, ws, l, boxes, st);
        default: return tile_boxes<3>(prob, opts, ws, l, boxes, st);
    }
}

// ---- forward summation for callers that cannot allocate ----------------------
//
// Some hosts cannot hand this library device memory: an XLA custom-call or
// plugin handler registered without a scratch allocator, a runtime whose
// device memory belongs entirely to another framework's pool, or a process
// with allocation forbidden once serving starts.  For them the FP32 forward
// takes its scratch from the fixed array below instead of a caller workspace.
// The array is part of the module: every GPU that loads the library holds it
// until the process exits.  In host code `sum32_static_scratch` only stands in
// for the symbol; the device address comes from cudaGetSymbolAddress, taken
// once per device on the first call made with that device current.
static __device__ __align__(256) unsigned char sum32_static_scratch[MSGB_SUM_F32_STATIC_SCRATCH_BYTES];

namespace {
constexpr int kMaxStaticDevices = 64;
std::mutex static_scratch_mu;
void *static_scratch_ptr[kMaxStaticDevices] = {};

int static_scratch_address(void **ptr) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(MSGB_ERR_CUDA, "msgb_sum_fwd_f32_static: cudaGetDevice: %s", cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxStaticDevices)
        return fail(MSGB_ERR_UNSUPPORTED, "msgb_sum_fwd_f32_static: device ordinal %d beyond %d", dev,
                    kMaxStaticDevices - 1);
    std::lock_guard<std::mutex> lock(static_scratch_mu);
    if (!static_scratch_ptr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, sum32_static_scratch);
        if (e != cudaSuccess || !p)
            return fail(MSGB_ERR_CUDA, "msgb_sum_fwd_f32_static: cudaGetSymbolAddress on device %d: %s", dev,
                        cudaGetErrorString(e));
        static_scratch_ptr[dev] = p;
    }
    *ptr = static_scratch_ptr[dev];
    return MSGB_OK;
}
}  // namespace

extern "C" int msgb_sum_fwd_f32_static(const msgb_problem *prob, const msgb_beam_set *beams,
                                       const msgb_sum_opts *opts, float *out, msgb_stream_t stream) {
    if (int e = validate_problem(prob)) return e;
    if (int e = validate_beams(prob, beams)) return e;
    if (!out) return fail(MSGB_ERR_ARG, "msgb_sum_fwd_f32_static: out is NULL");
    if (prob->nt == 0 || prob->ns == 0) return MSGB_OK;
    const Layout need = layout(prob, beams->n, false, tile_count(prob, opts));
    if (need.total > (size_t)MSGB_SUM_F32_STATIC_SCRATCH_BYTES)
        return fail(MSGB_ERR_UNSUPPORTED,
                    "msgb_sum_fwd_f32_static: %lld coefficients and %lld sensors need %zu bytes of scratch, more "
                    "than the %zu-byte static scratch; call msgb_sum_fwd_f32 with a workspace instead",
                    (long long)beams->n, (long long)prob->ns, need.total, (size_t)MSGB_SUM_F32_STATIC_SCRATCH_BYTES);
    cudaStream_t st = as_stream(stream);
    if (st) {
        // the array's address is per device: the stream must run on the current one
        int cur = 0, sdev = 0;
        cudaError_t e = cudaGetDevice(&cur);
        if (e == cudaSuccess) e = cudaStreamGetDevice(st, &sdev);
        if (e != cudaSuccess)
            return fail(MSGB_ERR_CUDA, "msgb_sum_fwd_f32_static: device of the stream: %s", cudaGetErrorString(e));
        if (sdev != cur)
            return fail(MSGB_ERR_ARG, "msgb_sum_fwd_f32_static: the stream belongs to device %d but device %d is current",
                        sdev, cur);
    }
    void *scratch = nullptr;
    if (int e = static_scratch_address(&scratch)) return e;
    Layout l;
    if (int e = check_ws(prob, beams, opts, false, scratch, MSGB_SUM_F32_STATIC_SCRATCH_BYTES, l)) return e;
    // Only the persistent kernel's work counter must start at zero; run_fwd
    // clears it on the stream before the launch.  Everything else in the
    // scratch is written by this call's preparation kernels before it is read.
    char *ws = (char *)scratch;
    switch (prob->ndim) {
        case 1: return run_fwd<1, false>(prob, beams, opts, ws, l, out, st, traj_src<1>(nullptr, nullptr, 1, 1));
        case 2: return run_fwd<2, false>(prob, beams, opts, ws, l, out, st, traj_src<2>(nullptr, nullptr, 1, 1));
        default: return run_fwd<3, false>(prob, beams, opts, ws, l, out, st, traj_src<3>(nullptr, nullptr, 1, 1));
    }
}
