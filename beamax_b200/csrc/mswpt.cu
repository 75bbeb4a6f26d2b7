// MSWPT tiling on the GPU: one global FFT (cuFFT, a library call) followed by
// per-level batched box kernels that fuse the dual-filter division, the window
// multiply, the parity roll, the unitary box IFFT (shared-memory radix-2), the
// IVP half-wave factor, the conjugate half-mask and the top_n key.
//
// Restates beamax transforms.py:591-733 (MSWPT.forward/_compute_coeffs) and
// :735-850 (MSWPT.inverse); the Hermitian adjoint of the forward is the
// inverse's structure with the forward's roll convention and a final division
// by sum g^2 (see the derivation next to msgb_mswpt_synthesis).
//
// Index conventions (per axis, N even, S even):
//   shifted Fourier index k in [0, N) <-> frequency k - N/2 (fftshift order);
//   unshifted FFT index u = (k + N/2) mod N;
//   patch element j of the box centred at c covers k = (c + N/2 - S/2 + j) mod N;
//   roll by r then ifftshift moves patch element j to q = (j - S/2 + r) mod S.
#include <cufft.h>

#include <vector>

#include "common.cuh"

struct msgb_mswpt {
    int nd;
    int N[3];
    int aspect[3];
    int red;
    int levels;
    int nbox;
    int64_t total;
    int64_t prodN;
    int64_t half_prodN;  // complex elements of the D2Z output
    // host copies of per-level metadata
    std::vector<int> bl;          // box_lengths
    std::vector<int> bshape;      // levels x nd (half supports)
    std::vector<int64_t> ccum;    // levels + 1
    std::vector<int> bcum;        // levels + 1
    std::vector<int> lat_cnt, lat_first, lat_step;  // levels x nd
    std::vector<int64_t> lat_off;                   // levels
    std::vector<int64_t> goff;                      // levels
    int max_patch;                                  // max prod S
    // device tables
    int32_t *d_centres = nullptr;
    int32_t *d_lattice = nullptr;
    double *d_gfilt = nullptr;
    double *d_ssq = nullptr;
    int64_t *d_ccum = nullptr;
    int32_t *d_bcum = nullptr;
    int32_t *d_bl = nullptr;
    int32_t *d_bshape = nullptr;
    cufftHandle plan_d2z = 0, plan_z2z = 0;
    size_t fft_work = 0;
};

namespace msgb {
namespace {

constexpr int THREADS = 256;

struct LevelArgs {
    int nd;
    int N[3];
    int S[3];        // support per axis
    int bhs[3];      // half support (box_shapes)
    int P;           // prod S
    int nbox;        // boxes at this level
    int box0;        // global id of the first box
    int64_t c0;      // coefficient offset of the level
    int64_t seg;     // coefficients in the level
    double inv_sqrtS;
};

LevelArgs level_args(const msgb_mswpt *p, int l) {
    LevelArgs a{};
    a.nd = p->nd;
    a.P = 1;
    for (int i = 0; i < 3; ++i) {
        a.N[i] = i < p->nd ? p->N[i] : 1;
        a.bhs[i] = i < p->nd ? p->bshape[l * p->nd + i] : 1;
        a.S[i] = i < p->nd ? 2 * a.bhs[i] : 1;
        a.P *= a.S[i];
    }
    a.nbox = p->bcum[l + 1] - p->bcum[l];
    a.box0 = p->bcum[l];
    a.c0 = p->ccum[l];
    a.seg = p->ccum[l + 1] - p->ccum[l];
    a.inv_sqrtS = 1.0 / sqrt((double)a.P);
    return a;
}

__device__ __forceinline__ int floordiv(int a, int b) {
    int q = a / b;
    if ((a % b != 0) && ((a < 0) != (b < 0))) --q;
    return q;
}
__device__ __forceinline__ int imod(int a, int b) {
    int r = a % b;
    return r < 0 ? r + b : r;
}

// In-place unitary-free radix-2 DFT along every axis of a (S0, S1, S2) complex
// array in shared memory; sign = +1 (inverse) or -1 (forward).  Twiddles are
// exp(sign 2 pi i m / S) from sincospi.
__device__ void smem_fft(double2 *x, const int *S, int nd, int sign, double2 *tw) {
    const int S0 = S[0], S1 = S[1], S2 = S[2];
    const int total = S0 * S1 * S2;
    for (int ax = 0; ax < nd; ++ax) {
        const int n = S[ax];
        if (n == 1) continue;
        const int stride = ax == 0 ? S1 * S2 : (ax == 1 ? S2 : 1);
        // twiddle table
        for (int m = threadIdx.x; m < n; m += blockDim.x) {
            double s, c;
            sincospi(2.0 * (double)m / (double)n, &s, &c);
            tw[m] = make_double2(c, sign * s);
        }
        int logn = 0;
        while ((1 << logn) < n) ++logn;
        // bit reversal along the axis
        for (int e = threadIdx.x; e < total; e += blockDim.x) {
            const int coord = (e / stride) % n;
            const int rev = __brev(coord) >> (32 - logn);
            if (rev > coord) {
                const int f = e + (rev - coord) * stride;
                double2 t = x[e];
                x[e] = x[f];
                x[f] = t;
            }
        }
        __syncthreads();
        for (int len = 2; len <= n; len <<= 1) {
            const int half = len >> 1;
            const int tstep = n / len;
            for (int bfly = threadIdx.x; bfly < total / 2; bfly += blockDim.x) {
                // decompose butterfly id into (line, position within line)
                const int pos = bfly % (n / 2);
                const int line = bfly / (n / 2);
                const int lo_idx = line % stride, hi_idx = line / stride;
                const int base = hi_idx * stride * n + lo_idx;
                const int grp = pos / half, k = pos % half;
                const int i0 = base + (grp * len + k) * stride;
                const int i1 = i0 + half * stride;
                const double2 w = tw[k * tstep];
                const double2 u = x[i0], v0 = x[i1];
                const double2 v = make_double2(v0.x * w.x - v0.y * w.y, v0.x * w.y + v0.y * w.x);
                x[i0] = make_double2(u.x + v.x, u.y + v.y);
                x[i1] = make_double2(u.x - v.x, u.y - v.y);
            }
            __syncthreads();
        }
    }
}

__device__ __forceinline__ void unravel(int e, const int *S, int *j) {
    j[2] = e % S[2];
    j[1] = (e / S[2]) % S[1];
    j[0] = e / (S[1] * S[2]);
}

// Read the unshifted spectrum value at index u (per axis), from either a full
// complex array or a D2Z half spectrum (last axis N/2 + 1) with Hermitian
// completion X[u] = conj(X[-u]).
__device__ __forceinline__ double2 read_spec(const double2 *X, int half, const int *N, int nd, const int *u) {
    if (!half) {
        int64_t idx = 0;
        for (int a = 0; a < nd; ++a) idx = idx * N[a] + u[a];
        return X[idx];
    }
    const int last = nd - 1;
    const int hl = N[last] / 2 + 1;
    int v[3] = {u[0], u[1], u[2]};
    bool cj = false;
    if (u[last] >= hl) {
        cj = true;
        for (int a = 0; a < nd; ++a) v[a] = (N[a] - u[a]) % N[a];
    }
    int64_t idx = 0;
    for (int a = 0; a < nd; ++a) idx = idx * (a == last ? hl : N[a]) + v[a];
    double2 r = X[idx];
    if (cj) r.y = -r.y;
    return r;
}

struct FwdArgs {
    const double2 *X;  // spectrum
    int half;          // X is a D2Z half spectrum
    int shifted;       // X is already in shifted order (Fourier input)
    double in_scale;   // 1/sqrt(prod N) for spatial input
    const double *ssq;
    const double *g;   // packed g of the level (prod S)
    const int32_t *centres;
    double scale;
    int half_mask;
    double2 *coeffs;
    double *keys;
};

__global__ void __launch_bounds__(THREADS) box_forward_kernel(LevelArgs L, FwdArgs A) {
    extern __shared__ double2 sm[];
    double2 *patch = sm;
    double2 *tw = sm + L.P;
    const int box = L.box0 + blockIdx.x;
    int cen[3] = {0, 0, 0}, r[3] = {0, 0, 0};
    for (int a = 0; a < L.nd; ++a) {
        cen[a] = A.centres[box * L.nd + a];
        // forward rolls: ((centre + N/2) + N/2) // bhs   (transforms.py:626,665-673)
        const int ri = floordiv(cen[a] + L.N[a] / 2 + L.N[a] / 2, L.bhs[a]);
        r[a] = (1 - 2 * (ri & 1)) * (L.bhs[a] / 2);
    }
    for (int e = threadIdx.x; e < L.P; e += blockDim.x) {
        int j[3];
        unravel(e, L.S, j);
        int k[3] = {0, 0, 0}, u[3] = {0, 0, 0}, q[3] = {0, 0, 0};
        int64_t kflat = 0;
        for (int a = 0; a < L.nd; ++a) {
            k[a] = imod(cen[a] + L.N[a] / 2 - L.S[a] / 2 + j[a], L.N[a]);
            u[a] = imod(k[a] + L.N[a] / 2, L.N[a]);
            q[a] = imod(j[a] - L.S[a] / 2 + r[a], L.S[a]);
            kflat = kflat * L.N[a] + k[a];
        }
        const double2 v = A.shifted ? A.X[kflat] : read_spec(A.X, A.half, L.N, L.nd, u);
        // unitary spectrum / sum g^2, then * g (transforms.py:731, :663)
        const double s = A.ssq[kflat], gv = A.g[e];
        const double2 w = make_double2(v.x * A.in_scale / s * gv, v.y * A.in_scale / s * gv);
        const int qf = (q[0] * L.S[1] + q[1]) * L.S[2] + q[2];
        patch[qf] = w;
    }
    __syncthreads();
    smem_fft(patch, L.S, L.nd, +1, tw);
    const int64_t base = L.c0 + (int64_t)blockIdx.x * L.P;
    for (int e = threadIdx.x; e < L.P; e += blockDim.x) {
        const int64_t loc = (int64_t)blockIdx.x * L.P + e;
        const double m = (!A.half_mask || loc < L.seg / 2) ? A.scale * L.inv_sqrtS : 0.0;
        const double2 v = patch[e];
        const double re = v.x * m, im = v.y * m;
        A.coeffs[base + e] = make_double2(re, im);
        if (A.keys) A.keys[base + e] = __dsqrt_rn(__dadd_rn(__dmul_rn(re, re), __dmul_rn(im, im)));
    }
}

struct SynArgs {
    const double2 *coeffs;
    const double *g;
    const int32_t *centres;
    int adjoint;       // forward roll convention
    double2 *contrib;  // per-box contributions, coefficient layout
};

// Per box: unitary FFT of the coefficient block, fftshift, unroll and window
// (transforms.py:826-837).
__global__ void __launch_bounds__(THREADS) box_synth_kernel(LevelArgs L, SynArgs A) {
    extern __shared__ double2 sm[];
    double2 *patch = sm;
    double2 *tw = sm + L.P;
    const int box = L.box0 + blockIdx.x;
    const int64_t base = L.c0 + (int64_t)blockIdx.x * L.P;
    for (int e = threadIdx.x; e < L.P; e += blockDim.x) patch[e] = A.coeffs[base + e];
    __syncthreads();
    smem_fft(patch, L.S, L.nd, -1, tw);
    int r[3] = {0, 0, 0};
    for (int a = 0; a < L.nd; ++a) {
        const int c = A.centres[box * L.nd + a];
        const int shift = A.adjoint ? L.N[a] : L.N[a] / 2;
        const int ri = floordiv(c + shift, L.bhs[a]);
        r[a] = (1 - 2 * (ri & 1)) * (L.bhs[a] / 2);
    }
    for (int e = threadIdx.x; e < L.P; e += blockDim.x) {
        int j[3];
        unravel(e, L.S, j);
        int q[3] = {0, 0, 0};
        for (int a = 0; a < L.nd; ++a) q[a] = imod(j[a] + r[a] + L.S[a] / 2, L.S[a]);
        const double2 v = patch[(q[0] * L.S[1] + q[1]) * L.S[2] + q[2]];
        const double s = A.g[e] * L.inv_sqrtS;
        A.contrib[base + e] = make_double2(v.x * s, v.y * s);
    }
}

struct GatherLevel {
    int cnt[3], first[3], step[3], S[3];
    int64_t lat_off;
    int box0;
    int64_t c0;
    int P;
};

struct GatherArgs {
    int nd, levels;
    int N[3];
    GatherLevel lv[8];
    const int32_t *lattice;
    const int32_t *centres;
    const double2 *contrib;
    const double *ssq;   // divide by sum g^2 (adjoint) when not NULL
    int fourier_out;     // write the shifted spectrum directly
    double out_scale;    // 1/sqrt(prod N)
    double2 *out;        // fourier_out: shifted order; else ifftshifted FFT input
};

// Deterministic synthesis gather: every Fourier bin sums the contributions of
// the boxes whose periodic support covers it, level by level in lattice order.
__global__ void __launch_bounds__(THREADS) synth_gather_kernel(GatherArgs A) {
    int64_t prodN = 1;
    for (int a = 0; a < A.nd; ++a) prodN *= A.N[a];
    const int64_t kf = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (kf >= prodN) return;
    int k[3] = {0, 0, 0};
    {
        int64_t rem = kf;
        for (int a = A.nd - 1; a >= 0; --a) {
            k[a] = (int)(rem % A.N[a]);
            rem /= A.N[a];
        }
    }
    double sr = 0.0, si = 0.0;
    for (int l = 0; l < A.levels; ++l) {
        const GatherLevel &G = A.lv[l];
        // candidate lattice indices per axis (at most 4 each)
        int cand[3][4], nc[3] = {1, 1, 1}, jj[3][4];
        cand[1][0] = cand[2][0] = 0;
        jj[1][0] = jj[2][0] = 0;
        bool none = false;
        for (int a = 0; a < A.nd; ++a) {
            nc[a] = 0;
            const int N = A.N[a], S = G.S[a], st = G.step[a];
            // box i covers k iff (k - (first + i st + N/2) + S/2) mod N < S
            const int z = imod(k[a] - N / 2 + S / 2 - G.first[a], N);
            // range 1: i st <= z, z - i st < S
            int ilo = floordiv(z - S, st) + 1, ihi = floordiv(z, st);
            if (ilo < 0) ilo = 0;
            if (ihi > G.cnt[a] - 1) ihi = G.cnt[a] - 1;
            for (int i = ilo; i <= ihi && nc[a] < 4; ++i) {
                cand[a][nc[a]] = i;
                jj[a][nc[a]] = z - i * st;
                nc[a]++;
            }
            // range 2: i st > z and z - i st + N < S
            ilo = floordiv(z + N - S, st) + 1;
            if (ilo <= ihi) ilo = ihi + 1;
            ihi = G.cnt[a] - 1;
            for (int i = ilo; i <= ihi && nc[a] < 4; ++i) {
                if (i * st <= z) continue;
                cand[a][nc[a]] = i;
                jj[a][nc[a]] = z - i * st + N;
                nc[a]++;
            }
            if (nc[a] == 0) none = true;
        }
        if (none) continue;
        for (int i0 = 0; i0 < nc[0]; ++i0)
            for (int i1 = 0; i1 < nc[1]; ++i1)
                for (int i2 = 0; i2 < nc[2]; ++i2) {
                    const int ci[3] = {cand[0][i0], cand[1][i1], cand[2][i2]};
                    const int cj[3] = {jj[0][i0], jj[1][i1], jj[2][i2]};
                    int64_t li = 0;
                    for (int a = 0; a < A.nd; ++a) li = li * G.cnt[a] + ci[a];
                    const int box = A.lattice[G.lat_off + li];
                    if (box < 0) continue;
                    int e = 0;
                    for (int a = 0; a < A.nd; ++a) e = e * G.S[a] + cj[a];
                    const double2 v = A.contrib[G.c0 + (int64_t)(box - G.box0) * G.P + e];
                    sr += v.x;
                    si += v.y;
                }
    }
    if (A.ssq) {
        const double s = A.ssq[kf];
        sr /= s;
        si /= s;
    }
    if (A.fourier_out) {
        A.out[kf] = make_double2(sr, si);
    } else {
        int64_t uf = 0;
        for (int a = 0; a < A.nd; ++a) uf = uf * A.N[a] + imod(k[a] + A.N[a] / 2, A.N[a]);
        A.out[uf] = make_double2(sr * A.out_scale, si * A.out_scale);
    }
}

__global__ void real_part_kernel(const double2 *in, int64_t n, double *out) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) out[i] = in[i].x;
}

__global__ void copy_complex_kernel(const double2 *in, int64_t n, double2 *out) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) out[i] = in[i];
}

size_t a256(size_t x) { return (x + 255) & ~size_t(255); }

struct WsLayout {
    size_t spec, contrib, fftwork, total;
};

WsLayout ws_layout(const msgb_mswpt *p) {
    WsLayout w{};
    size_t o = 0;
    w.spec = o;
    o = a256(o + sizeof(double2) * (size_t)p->prodN);
    w.contrib = o;
    o = a256(o + sizeof(double2) * (size_t)p->total);
    w.fftwork = o;
    o = a256(o + p->fft_work);
    w.total = o;
    return w;
}

int cufft_fail(const char *what, cufftResult r) { return fail(MSGB_ERR_CUDA, "%s: cuFFT error %d", what, (int)r); }

int smem_attr(const void *fn, size_t bytes) {
    if (bytes > 227 * 1024) return fail(MSGB_ERR_UNSUPPORTED, "box support too large for shared memory");
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) return fail(MSGB_ERR_CUDA, "cudaFuncSetAttribute: %s", cudaGetErrorString(e));
    return MSGB_OK;
}

}  // namespace
}  // namespace msgb

using namespace msgb;

extern "C" int msgb_mswpt_create(const msgb_mswpt_desc *d, msgb_mswpt **out) {
    if (!d || !out) return fail(MSGB_ERR_ARG, "msgb_mswpt_create: NULL argument");
    *out = nullptr;
    if (d->ndim < 1 || d->ndim > 3) return fail(MSGB_ERR_ARG, "ndim must be 1, 2 or 3");
    if (d->num_levels < 1 || d->num_levels > 8) return fail(MSGB_ERR_UNSUPPORTED, "1..8 levels supported");
    if (d->redundancy != 1 && d->redundancy != 2) return fail(MSGB_ERR_ARG, "redundancy must be 1 or 2");
    auto *p = new msgb_mswpt();
    p->nd = d->ndim;
    p->red = d->redundancy;
    p->levels = d->num_levels;
    p->nbox = d->total_boxes;
    p->prodN = 1;
    for (int a = 0; a < 3; ++a) {
        p->N[a] = a < d->ndim ? d->N[a] : 1;
        p->aspect[a] = a < d->ndim ? d->aspect[a] : 1;
        if (a < d->ndim && (p->N[a] <= 0 || p->N[a] % 2)) {
            delete p;
            return fail(MSGB_ERR_ARG, "N must be positive and even");
        }
        p->prodN *= p->N[a];
    }
    p->half_prodN = p->prodN / p->N[p->nd - 1] * (p->N[p->nd - 1] / 2 + 1);
    const int L = d->num_levels, nd = d->ndim;
    p->bl.assign(d->box_length, d->box_length + L);
    p->bshape.assign(d->box_shape, d->box_shape + L * nd);
    p->ccum.assign(d->coeffs_cumsum, d->coeffs_cumsum + L + 1);
    p->bcum.assign(d->boxes_cumsum, d->boxes_cumsum + L + 1);
    p->lat_cnt.assign(d->lattice_counts, d->lattice_counts + L * nd);
    p->lat_first.assign(d->lattice_first, d->lattice_first + L * nd);
    p->lat_step.assign(d->lattice_step, d->lattice_step + L * nd);
    p->lat_off.assign(d->lattice_offset, d->lattice_offset + L);
    p->goff.assign(d->gfilt_offset, d->gfilt_offset + L);
    p->total = p->ccum[L];
    p->max_patch = 1;
    int64_t gsize = 0, latsize = 0;
    for (int l = 0; l < L; ++l) {
        int P = 1, lat = 1;
        for (int a = 0; a < nd; ++a) {
            const int S = 2 * p->bshape[l * nd + a];
            if (S & (S - 1)) {
                delete p;
                return fail(MSGB_ERR_UNSUPPORTED, "box supports must be powers of two (got %d)", S);
            }
            P *= S;
            lat *= p->lat_cnt[l * nd + a];
        }
        if (P > p->max_patch) p->max_patch = P;
        gsize = p->goff[l] + P > gsize ? p->goff[l] + P : gsize;
        latsize = p->lat_off[l] + lat > latsize ? p->lat_off[l] + lat : latsize;
    }
    cudaError_t e = cudaSuccess;
    auto up = [&](void **dst, const void *src, size_t bytes) {
        if (e != cudaSuccess) return;
        e = cudaMalloc(dst, bytes > 0 ? bytes : 1);
        if (e == cudaSuccess && bytes) e = cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice);
    };
    up((void **)&p->d_centres, d->centres, sizeof(int32_t) * p->nbox * nd);
    up((void **)&p->d_lattice, d->lattice_box, sizeof(int32_t) * latsize);
    up((void **)&p->d_gfilt, d->gfilt, sizeof(double) * gsize);
    up((void **)&p->d_ssq, d->sum_gsquare, sizeof(double) * p->prodN);
    up((void **)&p->d_ccum, d->coeffs_cumsum, sizeof(int64_t) * (L + 1));
    up((void **)&p->d_bcum, d->boxes_cumsum, sizeof(int32_t) * (L + 1));
    up((void **)&p->d_bl, d->box_length, sizeof(int32_t) * L);
    up((void **)&p->d_bshape, d->box_shape, sizeof(int32_t) * L * nd);
    if (e != cudaSuccess) {
        msgb_mswpt_destroy(p);
        return fail(MSGB_ERR_CUDA, "msgb_mswpt_create: %s", cudaGetErrorString(e));
    }
    int n[3] = {p->N[0], p->N[1], p->N[2]};
    size_t w1 = 0, w2 = 0;
    cufftResult r = cufftCreate(&p->plan_d2z);
    if (r == CUFFT_SUCCESS) r = cufftSetAutoAllocation(p->plan_d2z, 0);
    if (r == CUFFT_SUCCESS) r = cufftMakePlanMany(p->plan_d2z, nd, n, nullptr, 1, 0, nullptr, 1, 0, CUFFT_D2Z, 1, &w1);
    if (r == CUFFT_SUCCESS) r = cufftCreate(&p->plan_z2z);
    if (r == CUFFT_SUCCESS) r = cufftSetAutoAllocation(p->plan_z2z, 0);
    if (r == CUFFT_SUCCESS) r = cufftMakePlanMany(p->plan_z2z, nd, n, nullptr, 1, 0, nullptr, 1, 0, CUFFT_Z2Z, 1, &w2);
    if (r != CUFFT_SUCCESS) {
        msgb_mswpt_destroy(p);
        return cufft_fail("msgb_mswpt_create", r);
    }
    p->fft_work = w1 > w2 ? w1 : w2;
    *out = p;
    return MSGB_OK;
}

extern "C" int msgb_mswpt_destroy(msgb_mswpt *p) {
    if (!p) return MSGB_OK;
    cudaFree(p->d_centres);
    cudaFree(p->d_lattice);
    cudaFree(p->d_gfilt);
    cudaFree(p->d_ssq);
    cudaFree(p->d_ccum);
    cudaFree(p->d_bcum);
    cudaFree(p->d_bl);
    cudaFree(p->d_bshape);
    if (p->plan_d2z) cufftDestroy(p->plan_d2z);
    if (p->plan_z2z) cufftDestroy(p->plan_z2z);
    delete p;
    return MSGB_OK;
}

extern "C" int64_t msgb_mswpt_total_coeffs(const msgb_mswpt *p) { return p ? p->total : -1; }

extern "C" size_t msgb_mswpt_workspace_size(const msgb_mswpt *p) { return p ? ws_layout(p).total : 0; }

static int check_ws(const msgb_mswpt *p, void *ws, size_t bytes) {
    if (!ws || bytes < ws_layout(p).total)
        return fail(MSGB_ERR_WORKSPACE, "MSWPT workspace too small: need %zu, got %zu", ws_layout(p).total, bytes);
    if (((uintptr_t)ws & 255) != 0) return fail(MSGB_ERR_WORKSPACE, "workspace must be 256-byte aligned");
    return MSGB_OK;
}

extern "C" int msgb_mswpt_forward(const msgb_mswpt *p, const double *in, int is_complex, int input_is_fourier,
                                  double scale, int apply_half_mask, double *coeffs, double *keys, void *workspace,
                                  size_t workspace_bytes, msgb_stream_t stream) {
    if (!p || !in || !coeffs) return fail(MSGB_ERR_ARG, "msgb_mswpt_forward: NULL argument");
    if (input_is_fourier && !is_complex) return fail(MSGB_ERR_ARG, "Fourier input must be complex");
    if (int e = check_ws(p, workspace, workspace_bytes)) return e;
    cudaStream_t st = as_stream(stream);
    const WsLayout w = ws_layout(p);
    char *ws = (char *)workspace;
    double2 *spec = (double2 *)(ws + w.spec);
    FwdArgs A{};
    A.half = 0;
    A.shifted = 0;
    A.in_scale = 1.0 / sqrt((double)p->prodN);
    if (input_is_fourier) {
        A.X = (const double2 *)in;
        A.shifted = 1;
        A.in_scale = 1.0;
    } else {
        cufftHandle h = is_complex ? p->plan_z2z : p->plan_d2z;
        cufftResult r = cufftSetStream(h, st);
        if (r == CUFFT_SUCCESS) r = cufftSetWorkArea(h, ws + w.fftwork);
        if (r == CUFFT_SUCCESS) {
            if (is_complex)
                r = cufftExecZ2Z(h, (cufftDoubleComplex *)in, (cufftDoubleComplex *)spec, CUFFT_FORWARD);
            else
                r = cufftExecD2Z(h, (cufftDoubleReal *)in, (cufftDoubleComplex *)spec);
        }
        if (r != CUFFT_SUCCESS) return cufft_fail("msgb_mswpt_forward", r);
        A.X = spec;
        A.half = is_complex ? 0 : 1;
    }
    A.ssq = p->d_ssq;
    A.centres = p->d_centres;
    A.scale = scale;
    A.half_mask = apply_half_mask;
    A.coeffs = (double2 *)coeffs;
    A.keys = keys;
    for (int l = 0; l < p->levels; ++l) {
        LevelArgs L = level_args(p, l);
        if (L.nbox == 0) continue;
        A.g = p->d_gfilt + p->goff[l];
        int maxS = 1;
        for (int a = 0; a < 3; ++a) maxS = L.S[a] > maxS ? L.S[a] : maxS;
        const size_t smem = sizeof(double2) * (L.P + maxS);
        if (int e = smem_attr((const void *)box_forward_kernel, smem)) return e;
        box_forward_kernel<<<L.nbox, THREADS, smem, st>>>(L, A);
    }
    return check_launch("msgb_mswpt_forward");
}

// Synthesis.  With W = (per box) unitary_ifft o roll(+r_fwd) o (g *) o extract
// o (/ sum g^2) o unitary_fft, the Hermitian adjoint is
//   W^H c = unitary_ifft( (1/sum g^2) * sum_boxes scatter( g * roll(unitary_fft(c_box), -r_fwd) ) ),
// which is MSWPT.inverse with the forward's roll convention and one extra
// division by sum g^2 (unitary_ifft^H = unitary_fft, roll^H = roll back,
// extract^H = periodic scatter-add; g and sum g^2 are real).
extern "C" int msgb_mswpt_synthesis(const msgb_mswpt *p, const double *coeffs, int mode, int real_output, double *out,
                                    void *workspace, size_t workspace_bytes, msgb_stream_t stream) {
    if (!p || !coeffs || !out) return fail(MSGB_ERR_ARG, "msgb_mswpt_synthesis: NULL argument");
    if (int e = check_ws(p, workspace, workspace_bytes)) return e;
    const int adjoint = mode & 1, fourier_out = (mode >> 1) & 1;
    cudaStream_t st = as_stream(stream);
    const WsLayout w = ws_layout(p);
    char *ws = (char *)workspace;
    double2 *spec = (double2 *)(ws + w.spec);
    double2 *contrib = (double2 *)(ws + w.contrib);
    SynArgs A{};
    A.coeffs = (const double2 *)coeffs;
    A.centres = p->d_centres;
    A.adjoint = adjoint;
    A.contrib = contrib;
    for (int l = 0; l < p->levels; ++l) {
        LevelArgs L = level_args(p, l);
        if (L.nbox == 0) continue;
        A.g = p->d_gfilt + p->goff[l];
        int maxS = 1;
        for (int a = 0; a < 3; ++a) maxS = L.S[a] > maxS ? L.S[a] : maxS;
        const size_t smem = sizeof(double2) * (L.P + maxS);
        if (int e = smem_attr((const void *)box_synth_kernel, smem)) return e;
        box_synth_kernel<<<L.nbox, THREADS, smem, st>>>(L, A);
    }
    GatherArgs G{};
    G.nd = p->nd;
    G.levels = p->levels;
    for (int a = 0; a < 3; ++a) G.N[a] = p->N[a];
    for (int l = 0; l < p->levels; ++l) {
        GatherLevel &gl = G.lv[l];
        gl.P = 1;
        for (int a = 0; a < 3; ++a) {
            const bool in = a < p->nd;
            gl.cnt[a] = in ? p->lat_cnt[l * p->nd + a] : 1;
            gl.first[a] = in ? p->lat_first[l * p->nd + a] : 0;
            gl.step[a] = in ? p->lat_step[l * p->nd + a] : 1;
            gl.S[a] = in ? 2 * p->bshape[l * p->nd + a] : 1;
            gl.P *= gl.S[a];
        }
        gl.lat_off = p->lat_off[l];
        gl.box0 = p->bcum[l];
        gl.c0 = p->ccum[l];
    }
    G.lattice = p->d_lattice;
    G.centres = p->d_centres;
    G.contrib = contrib;
    G.ssq = adjoint ? p->d_ssq : nullptr;
    G.fourier_out = fourier_out;
    G.out_scale = 1.0 / sqrt((double)p->prodN);
    G.out = (fourier_out && !real_output) ? (double2 *)out : spec;
    const unsigned blocks = (unsigned)((p->prodN + THREADS - 1) / THREADS);
    synth_gather_kernel<<<blocks, THREADS, 0, st>>>(G);
    if (int e = check_launch("msgb_mswpt_synthesis gather")) return e;
    if (!fourier_out) {
        cufftHandle h = p->plan_z2z;
        cufftResult r = cufftSetStream(h, st);
        if (r == CUFFT_SUCCESS) r = cufftSetWorkArea(h, ws + w.fftwork);
        if (r == CUFFT_SUCCESS) r = cufftExecZ2Z(h, (cufftDoubleComplex *)spec, (cufftDoubleComplex *)spec, CUFFT_INVERSE);
        if (r != CUFFT_SUCCESS) return cufft_fail("msgb_mswpt_synthesis", r);
        if (real_output)
            real_part_kernel<<<blocks, THREADS, 0, st>>>(spec, p->prodN, out);
        else
            copy_complex_kernel<<<blocks, THREADS, 0, st>>>(spec, p->prodN, (double2 *)out);
    } else if (real_output) {
        real_part_kernel<<<blocks, THREADS, 0, st>>>(spec, p->prodN, out);
    }
    return check_launch("msgb_mswpt_synthesis");
}

namespace msgb {
struct PlanView {
    int nd, red, levels;
    int N[3], aspect[3];
    int64_t ccum[9];
    int bcum[9];
    int bl[8];
    int bshape[8][3];
    const int32_t *centres;
};

int plan_view(const msgb_mswpt *p, PlanView &v) {
    if (!p) return fail(MSGB_ERR_ARG, "NULL MSWPT plan");
    v.nd = p->nd;
    v.red = p->red;
    v.levels = p->levels;
    for (int a = 0; a < 3; ++a) {
        v.N[a] = p->N[a];
        v.aspect[a] = p->aspect[a];
    }
    for (int l = 0; l <= p->levels; ++l) {
        v.ccum[l] = p->ccum[l];
        v.bcum[l] = p->bcum[l];
    }
    for (int l = 0; l < p->levels; ++l) {
        v.bl[l] = p->bl[l];
        for (int a = 0; a < 3; ++a) v.bshape[l][a] = a < p->nd ? p->bshape[l * p->nd + a] : 1;
    }
    v.centres = p->d_centres;
    return MSGB_OK;
}
}  // namespace msgb
