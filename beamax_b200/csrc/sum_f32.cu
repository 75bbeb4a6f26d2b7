// FP32 Gaussian-beam summation with Gaussian-cutoff culling, and its transpose.
//
// Same operator as compute_gaussian_beam_real (beamax gb/core.py:194-329)
// with solve_hom_diag (gb/gb_solvers.py:356-422), evaluated as
//   out(t, s) = sum_b 2|A_b(t)| cos(theta_b(t, s)) exp(-chi_b(t, s)),
//   theta = w (p.D + D^T Re M D / 2) + arg A,  chi = w D^T Im M D / 2,
//   D = s - x_b(t).
// Precision plan:
//  * sensors are grouped into spatially compact tiles (Morton order); each tile
//    has an FP64 anchor s0.  Per (beam, time) the large phase w p.(s0 - x(t)) +
//    arg A is formed in FP64 and reduced to [-pi, pi) before it meets FP32;
//    per sensor only w p.(s - s0) (bounded by the tile size) is FP32.
//  * evaluation is FP32 (MUFU exp2 / cos after explicit range reduction),
//    accumulation across beams is Kahan-compensated FP32.
// Culling: for a (beam, time tile, sensor tile) triple the exponent satisfies
//   chi >= (w/2) lambda_min(Im M(t)) |D|^2 >= (w/2) lam_lo(t_b) dist^2,
// with lam_lo(t) = 1 / (1/beta_min + (c t/|p|)^2 beta_max) (M0 = i diag(beta):
// Im M(t) = (S + R S^-1 R)^-1 with S = diag(1/beta), R = (c t/|p|) P_perp, so
// Im M is Loewner-decreasing in |t|) and dist the gap between the bounding
// boxes of the centre's path over the time tile and of the sensor tile.  A
// triple is skipped when that bound exceeds `cutoff` e-folds.
#include <cub/cub.cuh>

#include "common.cuh"

namespace msgb {
namespace {

constexpr int TS = 64;    // sensors per tile
constexpr int TT = 32;    // times per tile
constexpr int THREADS = 256;
constexpr int G = THREADS / TT;  // beams per record group
constexpr int SPT = TS / (THREADS / TT);  // sensors per thread (forward)
constexpr float kTwoPi = 6.283185307179586f;
constexpr float kInvTwoPi = 0.15915494309189535f;
constexpr float kLog2e = 1.4426950408889634f;

__device__ __forceinline__ float ex2_approx(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Reduce an FP32 angle to [-pi, pi] (bounded inputs, |theta| < 2^20).
__device__ __forceinline__ float reduce_angle(float th) {
    const float k = rintf(th * kInvTwoPi);
    return fmaf(-k, kTwoPi, th);
}

struct cf {
    float re, im;
};
__device__ __forceinline__ cf cmul(cf a, cf b) { return cf{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
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

// Per (beam, time) evaluation record.
template <int D>
struct Rec {
    float d0[D];                // s0 - x(t)
    float q[D * (D + 1) / 2];   // w/2 Re M (off-diagonals doubled)
    float e[D * (D + 1) / 2];   // -log2(e) w/2 Im M (off-diagonals doubled)
    float wp[D];                // w p
    float th0;                  // reduce(w p.(s0 - x(t)) + arg A)
    float amp;                  // 2 |A(t)|
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

// Closed-form beam state in FP32 (gb_solvers.py:306-353, :194-264) for the
// Hessian and the amplitude; the centre is formed in FP64 by the caller.
template <int D>
__device__ __forceinline__ void hom_mA_f32(const float *p0, const cf *al, cf a0, float c0t,
                                           cf *M, cf &A) {
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

template <int D>
__device__ __forceinline__ void make_rec(const ProbArgs &P, const BeamArgs &B, int64_t b, double t,
                                         const double *s0, Rec<D> &r) {
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
    double lin = 0.0;
    float p0f[D];
    cf al[D];
#pragma unroll
    for (int i = 0; i < D; ++i) {
        double x = B.x0[j * D + i] + c0 * (p0d[i] / np) * t;
        if (P.periodic[i]) x = pymod(x, P.L[i]);
        double d0 = s0[i] - x;
        if (P.periodic[i]) d0 -= P.L[i] * nearbyint(d0 / P.L[i]);
        r.d0[i] = (float)d0;
        lin = fma(w * p0d[i], d0, lin);
        r.wp[i] = (float)(w * p0d[i]);
        p0f[i] = (float)p0d[i];
        al[i] = cf{(float)B.alpha[2 * (j * D + i)], (float)B.alpha[2 * (j * D + i) + 1]};
    }
    cf M[D * (D + 1) / 2], A;
    hom_mA_f32<D>(p0f, al, cf{(float)B.a0[2 * j], (float)B.a0[2 * j + 1]}, (float)(c0 * t), M, A);
    const float wf = (float)w;
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
        for (int k = i; k < D; ++k) {
            const int q = sym_index<D>(i, k);
            const float f = (i == k ? 0.5f : 1.0f) * wf;
            r.q[q] = f * M[q].re;
            r.e[q] = -kLog2e * f * M[q].im;
        }
    float re = A.re;
    if (A.re == 0.0f && A.im == 0.0f) re = 1e-12f;
    const double th = lin + (double)atan2f(A.im, re);
    r.th0 = (float)(th - 6.283185307179586 * nearbyint(th * 0.15915494309189535));
    r.amp = 2.0f * sqrtf(fmaf(A.re, A.re, A.im * A.im));
}

template <int D>
__device__ __forceinline__ bool survives(const Cull<D> &cb, float c0, float ta, float tb,
                                         const TileInfo<D> &ti, const ProbArgs &P, float cutoff) {
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
template <int D>
__global__ void morton_kernel(const double *sens, int64_t ns, ProbArgs P, uint32_t *key, int32_t *val) {
    const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (s >= ns) return;
    const int bits = D == 1 ? 31 : (D == 2 ? 16 : 10);
    uint32_t q[D];
#pragma unroll
    for (int i = 0; i < D; ++i) {
        double u = sens[s * D + i] / P.L[i];
        u = fmin(fmax(u, 0.0), 1.0 - 1e-12);
        q[i] = (uint32_t)(u * (double)(1u << bits));
    }
    uint32_t k = 0;
    for (int b = bits - 1; b >= 0; --b)
#pragma unroll
        for (int i = 0; i < D; ++i) k = (k << 1) | ((q[i] >> b) & 1u);
    key[s] = k;
    val[s] = (int32_t)s;
}

template <int D>
__global__ void tile_kernel(const double *sens, int64_t ns, const int32_t *perm, TileInfo<D> *tiles,
                            float *ds, double *sorted) {
    const int64_t tile = blockIdx.x;
    const int64_t first = tile * TS;
    const int64_t cnt = min((int64_t)TS, ns - first);
    __shared__ double lo[D], hi[D];
    if (threadIdx.x == 0) {
        for (int i = 0; i < D; ++i) {
            double a = 1e300, b = -1e300;
            for (int64_t k = 0; k < cnt; ++k) {
                const double v = sens[(int64_t)perm[first + k] * D + i];
                a = fmin(a, v);
                b = fmax(b, v);
            }
            lo[i] = a;
            hi[i] = b;
            tiles[tile].s0[i] = 0.5 * (a + b);
            tiles[tile].lo[i] = (float)a;
            tiles[tile].hi[i] = (float)b;
        }
    }
    __syncthreads();
    for (int64_t k = threadIdx.x; k < cnt; k += blockDim.x) {
        for (int i = 0; i < D; ++i) {
            const double v = sens[(int64_t)perm[first + k] * D + i];
            ds[(first + k) * D + i] = (float)(v - 0.5 * (lo[i] + hi[i]));
            sorted[(first + k) * D + i] = v;
        }
    }
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

__global__ void permute_rows_kernel(const float *data, const int32_t *perm, int64_t nt, int64_t ns, float *out) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= nt * ns) return;
    const int64_t t = i / ns, s = i - t * ns;
    out[i] = data[t * ns + perm[s]];
}

// ------------------------------------------------------------------ forward
template <int D>
__global__ void __launch_bounds__(THREADS) fwd32_kernel(ProbArgs P, BeamArgs B, const Cull<D> *cull,
                                                        const TileInfo<D> *tiles, const float *ds,
                                                        const int32_t *perm, float cutoff, float *out,
                                                        unsigned long long *eval_count) {
    __shared__ Rec<D> recs[G * TT];
    __shared__ int64_t surv[THREADS * 2];
    __shared__ int nsurv_s;
    __shared__ int warp_cnt[THREADS / 32];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int64_t st = blockIdx.x, tt = blockIdx.y;
    const int64_t s_first = st * TS, t_first = tt * TT;
    const int s_cnt = (int)min((int64_t)TS, P.ns - s_first);
    const int t_cnt = (int)min((int64_t)TT, P.nt - t_first);
    const TileInfo<D> ti = tiles[st];
    const float ta = (float)P.ts[t_first], tb = (float)P.ts[t_first + t_cnt - 1];

    const int tl = tid / (THREADS / TT);   // my time in the tile
    const int sl = tid % (THREADS / TT);   // my sensor lane
    float dsx[SPT][D];
#pragma unroll
    for (int k = 0; k < SPT; ++k) {
        const int s = sl + k * (THREADS / TT);
#pragma unroll
        for (int i = 0; i < D; ++i) dsx[k][i] = s < s_cnt ? ds[(s_first + s) * D + i] : 0.0f;
    }
    float acc[SPT], cmp[SPT];
#pragma unroll
    for (int k = 0; k < SPT; ++k) acc[k] = 0.0f, cmp[k] = 0.0f;
    unsigned long long evals = 0;

    for (int64_t j0 = 0; j0 < B.n; j0 += THREADS) {
        // 1. cull both modes of THREADS coefficients.
        const int64_t j = j0 + tid;
        bool keep_p = false, keep_m = false;
        if (j < B.n) {
            const Cull<D> cb = cull[j];
            keep_p = survives<D>(cb, (float)P.c, ta, tb, ti, P, cutoff);
            keep_m = survives<D>(cb, -(float)P.c, ta, tb, ti, P, cutoff);
        }
        const unsigned bp = __ballot_sync(0xffffffffu, keep_p);
        const unsigned bm = __ballot_sync(0xffffffffu, keep_m);
        if (lane == 0) warp_cnt[warp] = __popc(bp) + __popc(bm);
        __syncthreads();
        int off = 0, tot = 0;
        for (int w = 0; w < THREADS / 32; ++w) {
            if (w < warp) off += warp_cnt[w];
            tot += warp_cnt[w];
        }
        const unsigned lt = (1u << lane) - 1u;
        if (keep_p) surv[off + __popc(bp & lt)] = j;
        if (keep_m) surv[off + __popc(bp) + __popc(bm & lt)] = j + B.n;
        if (tid == 0) nsurv_s = tot;
        __syncthreads();
        const int nsurv = nsurv_s;
        evals += (unsigned long long)nsurv;
        // 2. evaluate survivors in groups of G beams x TT times.
        for (int g0 = 0; g0 < nsurv; g0 += G) {
            {
                const int gl = tid / TT, tloc = tid % TT;
                Rec<D> &r = recs[gl * TT + tloc];
                if (g0 + gl < nsurv && tloc < t_cnt) {
                    make_rec<D>(P, B, surv[g0 + gl], P.ts[t_first + tloc], ti.s0, r);
                } else {
                    r.amp = 0.0f;
                    r.th0 = 0.0f;
#pragma unroll
                    for (int i = 0; i < D; ++i) r.d0[i] = 0.0f, r.wp[i] = 0.0f;
#pragma unroll
                    for (int q = 0; q < D * (D + 1) / 2; ++q) r.q[q] = 0.0f, r.e[q] = 0.0f;
                }
            }
            __syncthreads();
            const int ng = min(G, nsurv - g0);
            for (int gl = 0; gl < ng; ++gl) {
                const Rec<D> r = recs[gl * TT + tl];
#pragma unroll
                for (int k = 0; k < SPT; ++k) {
                    float Dl[D];
                    float th = r.th0;
#pragma unroll
                    for (int i = 0; i < D; ++i) {
                        Dl[i] = dsx[k][i] + r.d0[i];
                        if (P.periodic[i]) Dl[i] -= (float)P.L[i] * rintf(Dl[i] / (float)P.L[i]);
                        th = fmaf(r.wp[i], dsx[k][i], th);
                    }
                    float ex = 0.0f;
#pragma unroll
                    for (int i = 0; i < D; ++i)
#pragma unroll
                        for (int m = i; m < D; ++m) {
                            const int q = sym_index<D>(i, m);
                            const float dd = Dl[i] * Dl[m];
                            th = fmaf(r.q[q], dd, th);
                            ex = fmaf(r.e[q], dd, ex);
                        }
                    const float v = r.amp * __cosf(reduce_angle(th)) * ex2_approx(ex);
                    // Kahan-compensated accumulation across beams.
                    const float y = v - cmp[k];
                    const float tsum = acc[k] + y;
                    cmp[k] = (tsum - acc[k]) - y;
                    acc[k] = tsum;
                }
            }
            __syncthreads();
        }
    }
    if (tl < t_cnt) {
        const int64_t t = t_first + tl;
#pragma unroll
        for (int k = 0; k < SPT; ++k) {
            const int s = sl + k * (THREADS / TT);
            if (s < s_cnt) out[t * P.ns + perm[s_first + s]] = acc[k] - cmp[k];
        }
    }
    if (eval_count && tid == 0 && evals)
        atomicAdd(eval_count, evals * (unsigned long long)t_cnt * (unsigned long long)s_cnt);
}

// ------------------------------------------------------------------ adjoint
// One warp per selected coefficient (both modes).  Lanes test 32 sensor tiles
// at a time, build 32 per-time records for a surviving tile in shared memory,
// then evaluate two sensors each over the tile's times.
template <int D>
__global__ void __launch_bounds__(THREADS) adj32_kernel(ProbArgs P, BeamArgs B, const Cull<D> *cull,
                                                        const TileInfo<D> *tiles, const float *ds,
                                                        const float *data_sorted, float cutoff,
                                                        double *g, unsigned long long *eval_count) {
    __shared__ Rec<D> recs_all[THREADS / 32][TT];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t j = (int64_t)blockIdx.x * (THREADS / 32) + warp;
    if (j >= B.n) return;
    Rec<D> *recs = recs_all[warp];
    const Cull<D> cb = cull[j];
    const int64_t n_st = (P.ns + TS - 1) / TS, n_tt = (P.nt + TT - 1) / TT;
    double gre = 0.0, gim = 0.0;
    unsigned long long evals = 0;
    for (int m = 0; m < 2; ++m) {
        const float c0 = m == 0 ? (float)P.c : -(float)P.c;
        const int64_t b = m == 0 ? j : j + B.n;
        for (int64_t tt = 0; tt < n_tt; ++tt) {
            const int64_t t_first = tt * TT;
            const int t_cnt = (int)min((int64_t)TT, P.nt - t_first);
            const float ta = (float)P.ts[t_first], tb = (float)P.ts[t_first + t_cnt - 1];
            for (int64_t st0 = 0; st0 < n_st; st0 += 32) {
                const int64_t st_l = st0 + lane;
                const bool keep = st_l < n_st && survives<D>(cb, c0, ta, tb, tiles[st_l], P, cutoff);
                unsigned mask = __ballot_sync(0xffffffffu, keep);
                while (mask) {
                    const int k = __ffs(mask) - 1;
                    mask &= mask - 1;
                    const int64_t st = st0 + k;
                    const int64_t s_first = st * TS;
                    const int s_cnt = (int)min((int64_t)TS, P.ns - s_first);
                    const TileInfo<D> ti = tiles[st];
                    __syncwarp();
                    if (lane < t_cnt) make_rec<D>(P, B, b, P.ts[t_first + lane], ti.s0, recs[lane]);
                    __syncwarp();
                    float pr = 0.0f, pi = 0.0f;
#pragma unroll
                    for (int h = 0; h < TS / 32; ++h) {
                        const int s = lane + 32 * h;
                        if (s >= s_cnt) continue;
                        float dsl[D];
#pragma unroll
                        for (int i = 0; i < D; ++i) dsl[i] = ds[(s_first + s) * D + i];
                        const float *dcol = data_sorted + s_first + s;
                        for (int tl = 0; tl < t_cnt; ++tl) {
                            const Rec<D> &r = recs[tl];
                            float Dl[D];
                            float th = r.th0;
#pragma unroll
                            for (int i = 0; i < D; ++i) {
                                Dl[i] = dsl[i] + r.d0[i];
                                if (P.periodic[i]) Dl[i] -= (float)P.L[i] * rintf(Dl[i] / (float)P.L[i]);
                                th = fmaf(r.wp[i], dsl[i], th);
                            }
                            float ex = 0.0f;
#pragma unroll
                            for (int i = 0; i < D; ++i)
#pragma unroll
                                for (int q2 = i; q2 < D; ++q2) {
                                    const int q = sym_index<D>(i, q2);
                                    const float dd = Dl[i] * Dl[q2];
                                    th = fmaf(r.q[q], dd, th);
                                    ex = fmaf(r.e[q], dd, ex);
                                }
                            float sn, cs;
                            __sincosf(reduce_angle(th), &sn, &cs);
                            const float v = dcol[(t_first + tl) * P.ns] * r.amp * ex2_approx(ex);
                            pr = fmaf(v, cs, pr);
                            pi = fmaf(-v, sn, pi);
                        }
                    }
                    gre += (double)pr;
                    gim += (double)pi;
                    evals += (unsigned long long)t_cnt * (unsigned long long)s_cnt;
                }
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        gre += __shfl_down_sync(0xffffffffu, gre, o);
        gim += __shfl_down_sync(0xffffffffu, gim, o);
    }
    if (lane == 0) {
        g[2 * j] = gre;
        g[2 * j + 1] = gim;
        if (eval_count && evals) atomicAdd(eval_count, evals);
    }
}

// ------------------------------------------------------------------ workspace
struct Layout {
    size_t keys_in, keys_out, vals_in, vals_out, cub, tiles, ds, sorted, cull, data, total;
    size_t cub_bytes;
};

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

Layout layout(const msgb_problem *p, int64_t n_beams, bool with_data) {
    Layout l{};
    const int D = p->ndim;
    const int64_t ns = p->ns;
    const int64_t n_st = (ns + TS - 1) / TS;
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
    l.ds = o; o = align256(o + ns * D * 4);
    l.sorted = o; o = align256(o + ns * D * 8);
    l.cull = o; o = align256(o + (n_beams > 0 ? n_beams : 1) * sizeof(Cull<3>));
    l.data = o; o = align256(o + (with_data ? p->nt * ns * 4 : 0));
    l.total = o;
    return l;
}

template <int D>
int prep(const msgb_problem *p, const msgb_beam_set *b, const Layout &l, char *ws, cudaStream_t st) {
    const int64_t ns = p->ns;
    uint32_t *kin = (uint32_t *)(ws + l.keys_in), *kout = (uint32_t *)(ws + l.keys_out);
    int32_t *vin = (int32_t *)(ws + l.vals_in), *vout = (int32_t *)(ws + l.vals_out);
    const int blk = 256;
    morton_kernel<D><<<(unsigned)((ns + blk - 1) / blk), blk, 0, st>>>(p->sensors, ns, to_args(p), kin, vin);
    size_t cb = l.cub_bytes;
    cub::DeviceRadixSort::SortPairs(ws + l.cub, cb, kin, kout, vin, vout, (int)ns, 0, 32, st);
    const int64_t n_st = (ns + TS - 1) / TS;
    tile_kernel<D><<<(unsigned)n_st, 64, 0, st>>>(p->sensors, ns, vout, (TileInfo<D> *)(ws + l.tiles),
                                                 (float *)(ws + l.ds), (double *)(ws + l.sorted));
    if (b->n > 0)
        cull_prep_kernel<D><<<(unsigned)((b->n + blk - 1) / blk), blk, 0, st>>>(to_args(b), (Cull<D> *)(ws + l.cull));
    return check_launch("msgb sum f32 prep");
}

template <int D>
int run_fwd(const msgb_problem *p, const msgb_beam_set *b, const msgb_sum_opts *o, char *ws,
            const Layout &l, float *out, cudaStream_t st) {
    if (int e = prep<D>(p, b, l, ws, st)) return e;
    const int64_t n_st = (p->ns + TS - 1) / TS, n_tt = (p->nt + TT - 1) / TT;
    if (n_tt > 65535) return fail(MSGB_ERR_UNSUPPORTED, "msgb_sum_fwd_f32: nt too large");
    dim3 grid((unsigned)n_st, (unsigned)n_tt);
    ProbArgs P = to_args(p);
    P.sensors = (const double *)(ws + l.sorted);
    fwd32_kernel<D><<<grid, THREADS, 0, st>>>(P, to_args(b), (const Cull<D> *)(ws + l.cull),
                                               (const TileInfo<D> *)(ws + l.tiles), (const float *)(ws + l.ds),
                                               (const int32_t *)(ws + l.vals_out), o ? (float)o->cutoff : 0.0f,
                                               out, o ? o->eval_count : nullptr);
    return check_launch("msgb_sum_fwd_f32");
}

template <int D>
int run_adj(const msgb_problem *p, const msgb_beam_set *b, const msgb_sum_opts *o, char *ws,
            const Layout &l, const float *data, double *g, cudaStream_t st) {
    if (int e = prep<D>(p, b, l, ws, st)) return e;
    const int64_t tot = p->nt * p->ns;
    permute_rows_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(data, (const int32_t *)(ws + l.vals_out),
                                                                     p->nt, p->ns, (float *)(ws + l.data));
    ProbArgs P = to_args(p);
    P.sensors = (const double *)(ws + l.sorted);
    const unsigned grid = (unsigned)((b->n + THREADS / 32 - 1) / (THREADS / 32));
    adj32_kernel<D><<<grid, THREADS, 0, st>>>(P, to_args(b), (const Cull<D> *)(ws + l.cull),
                                               (const TileInfo<D> *)(ws + l.tiles), (const float *)(ws + l.ds),
                                               (const float *)(ws + l.data), o ? (float)o->cutoff : 0.0f, g,
                                               o ? o->eval_count : nullptr);
    return check_launch("msgb_adj_gather_f32");
}

}  // namespace
}  // namespace msgb

using namespace msgb;

extern "C" size_t msgb_sum_f32_workspace_size(const msgb_problem *prob, int64_t n) {
    if (validate_problem(prob) || n < 0) return 0;
    return layout(prob, n, true).total;
}

static int check_ws(const msgb_problem *p, const msgb_beam_set *b, bool with_data, void *ws, size_t bytes,
                    Layout &l) {
    l = layout(p, b->n, with_data);
    if (b->n > (int64_t(1) << 22)) return fail(MSGB_ERR_UNSUPPORTED, "at most 2^22 selected coefficients");
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
    if (int e = check_ws(prob, beams, false, workspace, workspace_bytes, l)) return e;
    cudaStream_t st = as_stream(stream);
    char *ws = (char *)workspace;
    switch (prob->ndim) {
        case 1: return run_fwd<1>(prob, beams, opts, ws, l, out, st);
        case 2: return run_fwd<2>(prob, beams, opts, ws, l, out, st);
        default: return run_fwd<3>(prob, beams, opts, ws, l, out, st);
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
    if (int e = check_ws(prob, beams, true, workspace, workspace_bytes, l)) return e;
    cudaStream_t st = as_stream(stream);
    char *ws = (char *)workspace;
    switch (prob->ndim) {
        case 1: return run_adj<1>(prob, beams, opts, ws, l, data, g, st);
        case 2: return run_adj<2>(prob, beams, opts, ws, l, data, g, st);
        default: return run_adj<3>(prob, beams, opts, ws, l, data, g, st);
    }
}
