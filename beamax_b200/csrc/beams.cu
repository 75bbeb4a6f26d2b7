// top_n selection, beam initialisation and the coefficient-space scatter of
// the transpose.
//
// top_n restates forward_solver_utils.py:65-89 with jnp.argpartition's tie
// rule: keys are the IEEE bit patterns of sqrt(re*re + im*im) (monotone for
// non-negative doubles); a stable ascending radix sort of (key, index) pairs
// orders them by (key, index) and the last n entries are the selection, in the
// order the reference returns them (increasing magnitude, ties by index).
//
// Beam init restates compute_forward_parameters (forward_solver_utils.py:
// 255-373), compute_frame_phase (transforms.py:193-226) and
// _coefficient_positions (forward_solver_utils.py:233-252).
#include <cub/cub.cuh>

#include "traj.cuh"

// Layout shared with mswpt.cu (only the fields read here).
struct msgb_mswpt;

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
int plan_view(const msgb_mswpt *p, PlanView &v);
}  // namespace msgb

namespace msgb {
namespace {

__global__ void key_bits_kernel(const double *keys, int64_t n, uint64_t *kb, int32_t *idx) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    double k = keys[i];
    if (k == 0.0) k = 0.0;  // fold -0.0 onto +0.0
    kb[i] = (uint64_t)__double_as_longlong(k);
    idx[i] = (int32_t)i;
}

__global__ void take_last_kernel(const int32_t *sorted_idx, int64_t total, int64_t n, const double2 *coeffs,
                                 int64_t *idx_out, double2 *val_out) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t j = sorted_idx[total - n + i];
    idx_out[i] = j;
    if (val_out) val_out[i] = coeffs[j];
}

__device__ __forceinline__ int floordiv(int a, int b) {
    int q = a / b;
    if ((a % b != 0) && ((a < 0) != (b < 0))) --q;
    return q;
}

struct InitArgs {
    PlanView v;
    double L[3];
    const int64_t *idx;
    const double2 *values;
    int64_t n;
    msgb_beam_out out;
};

__global__ void beam_init_kernel(InitArgs A) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= A.n) return;
    const PlanView &v = A.v;
    const int nd = v.nd;
    const int64_t flat = A.idx[i];
    // level = searchsorted(cumsum(prod shapes), flat, 'right')
    int l = 0;
    while (l < v.levels - 1 && flat >= v.ccum[l + 1]) ++l;
    const int64_t local = flat - v.ccum[l];
    int S[3] = {1, 1, 1};
    int64_t P = 1;
    for (int a = 0; a < nd; ++a) {
        S[a] = 2 * v.bshape[l][a];
        P *= S[a];
    }
    const int64_t box_local = local / P;
    int64_t rem = local - box_local * P;
    int k[3] = {0, 0, 0};
    for (int a = nd - 1; a >= 0; --a) {
        k[a] = (int)(rem % S[a]);
        rem /= S[a];
    }
    const int64_t box = v.bcum[l] + box_local;
    double cen[3], norm2 = 0.0;
    int ci[3];
    for (int a = 0; a < nd; ++a) {
        ci[a] = v.centres[box * nd + a];
        cen[a] = (double)ci[a] / A.L[a];
        norm2 += cen[a] * cen[a];
    }
    const double norm = sqrt(norm2);
    const double pi = 3.141592653589793;
    double a0 = 1.0, cycles = 0.0;
    for (int a = 0; a < nd; ++a) {
        const double bl = (double)v.bl[l] / A.L[a] * (double)v.aspect[a];
        const double Ll = bl * v.red;
        const double sig = bl / 2.0;
        const double ps = pi * sig;
        A.out.p0[i * nd + a] = 2.0 * pi * cen[a] / norm;
        A.out.alpha[2 * (i * nd + a)] = 0.0;
        A.out.alpha[2 * (i * nd + a) + 1] = 2.0 * (ps * ps) / norm;
        a0 *= sqrt((pi * A.L[a]) / (Ll * (double)v.N[a])) * sig;
        // frame phase (transforms.py:207-226)
        const int support = v.bl[l] * v.red * v.aspect[a];
        const int half = support / 2;
        const int parity = floordiv(ci[a] + v.N[a] / 2, half);
        const int sign = 1 - 2 * (parity & 1);
        const int rolls = sign * (half / 2);
        cycles += (double)(ci[a] - rolls) * (double)k[a] / (double)support;
        // _coefficient_positions (forward_solver_utils.py:233-252)
        A.out.x0[i * nd + a] = (double)k[a] * A.L[a] / (double)support;
    }
    cycles = cycles - floor(cycles);  // jnp.remainder(., 1.0)
    double s, c;
    sincospi(2.0 * cycles, &s, &c);
    cd au = cd{a0 * c, a0 * s};
    if (A.out.a0_unit) {
        A.out.a0_unit[2 * i] = au.re;
        A.out.a0_unit[2 * i + 1] = au.im;
    }
    cd val = A.values ? cd{A.values[i].x, A.values[i].y} : cd{1.0, 0.0};
    cd a = au * val;
    A.out.a0[2 * i] = a.re;
    A.out.a0[2 * i + 1] = a.im;
    A.out.omega[i] = norm;
}

// compute_coefficients with an initial time derivative
// (forward_solver_utils.py:716-786): c = 0.5 (a + branch i b / vg) with
// vg = G(x_b, p_b, +1) = c(x_b) |p_b| (gb_utils.py:11-44), x_b the
// coefficient's position (_coefficient_positions) and p_b = 2 pi centre / L
// its box's centre frequency.
struct DpdtArgs {
    PlanView v;
    double L[3];
    MediumArgs med;
    const double2 *a, *b;
    int64_t total;
    double branch;
    int mask;
    double2 *out;
    double *keys;
};

template <int D>
__global__ void dpdt_kernel(DpdtArgs A) {
    const int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (f >= A.total) return;
    const PlanView &v = A.v;
    int l = 0;
    while (l < v.levels - 1 && f >= v.ccum[l + 1]) ++l;
    const int64_t local = f - v.ccum[l];
    int S[3] = {1, 1, 1};
    int64_t P = 1;
    for (int a = 0; a < D; ++a) {
        S[a] = 2 * v.bshape[l][a];
        P *= S[a];
    }
    const int64_t box_local = local / P;
    int64_t rem = local - box_local * P;
    int k[3] = {0, 0, 0};
    for (int a = D - 1; a >= 0; --a) {
        k[a] = (int)(rem % S[a]);
        rem /= S[a];
    }
    const int64_t box = v.bcum[l] + box_local;
    double x[D], p2 = 0.0;
    for (int a = 0; a < D; ++a) {
        const int support = v.bl[l] * v.red * v.aspect[a];
        x[a] = (double)k[a] * A.L[a] / (double)support;
        const double pb = 2.0 * 3.141592653589793 * (double)v.centres[box * D + a] / A.L[a];
        p2 += pb * pb;
    }
    double c, g[D], H[D * D];
    speed_eval<D>(A.med, x, c, g, H);
    const double vg = c * sqrt(p2);
    const double2 ca = A.a[f], cb = A.b[f];
    // i b / vg = (-b.im, b.re) / vg
    double re = 0.5 * (ca.x - A.branch * cb.y / vg);
    double im = 0.5 * (ca.y + A.branch * cb.x / vg);
    if (A.mask && local >= (v.ccum[l + 1] - v.ccum[l]) / 2) re = im = 0.0;
    A.out[f] = make_double2(re, im);
    if (A.keys) A.keys[f] = sqrt(__dadd_rn(__dmul_rn(re, re), __dmul_rn(im, im)));
}

// compute_TR_parameters (tr_solver_utils.py:205-440) for one selected
// coefficient of the boundary-data transform.
struct TrInitArgs {
    PlanView v;
    double L[3];
    msgb_tr_geometry geo;
    MediumArgs med;
    const int64_t *idx;
    const double2 *values;
    int64_t n;
    int b_inverse;
    double guard;
    msgb_tr_beams out;
};

template <int D>
__global__ void tr_init_kernel(TrInitArgs A) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= A.n) return;
    const PlanView &v = A.v;
    const double pi = 3.141592653589793;
    const int64_t flat = A.idx[i];
    int l = 0;
    while (l < v.levels - 1 && flat >= v.ccum[l + 1]) ++l;
    const int64_t local = flat - v.ccum[l];
    int S[3] = {1, 1, 1};
    int64_t P = 1;
    for (int a = 0; a < D; ++a) {
        S[a] = 2 * v.bshape[l][a];
        P *= S[a];
    }
    const int64_t box_local = local / P;
    int64_t rem = local - box_local * P;
    int k[3] = {0, 0, 0};
    for (int a = D - 1; a >= 0; --a) {
        k[a] = (int)(rem % S[a]);
        rem /= S[a];
    }
    const int64_t box = v.bcum[l] + box_local;
    double ch[D], Lls[D], sig[D], ats = 1.0, cycles = 0.0;
    for (int a = 0; a < D; ++a) {
        const int ci = v.centres[box * D + a];
        ch[a] = (double)ci / A.L[a];
        const double bl = (double)v.bl[l] / A.L[a] * (double)v.aspect[a];
        Lls[a] = bl * v.red;
        sig[a] = bl / 2.0;
        ats *= sqrt((pi * A.L[a]) / (Lls[a] * (double)v.N[a])) * sig[a];
        const int support = v.bl[l] * v.red * v.aspect[a];
        const int half = support / 2;
        const int parity = floordiv(ci + v.N[a] / 2, half);
        const int sgn = 1 - 2 * (parity & 1);
        const int rolls = sgn * (half / 2);
        cycles += (double)(ci - rolls) * (double)k[a] / (double)support;
    }
    cycles = cycles - floor(cycles);
    double ps, pc;
    sincospi(2.0 * cycles, &ps, &pc);
    const double tau = ch[0];
    const double signum = tau > 0.0 ? -1.0 : (tau < 0.0 ? 1.0 : 0.0);
    const double omega = fmax(fabs(tau), 1e-6);
    const double t0 = (double)k[0] / Lls[0];
    // position on the detector: normal axis fixed, tangential axes in order
    const int na = A.geo.normal_axis;
    double x[D];
    int j = 0;
    for (int a = 0; a < D; ++a) {
        if (a == na) {
            x[a] = A.geo.normal_value;
        } else {
            x[a] = (double)k[1 + j] / Lls[1 + j];
            ++j;
        }
    }
    double c, g[D], H[D * D];
    speed_eval<D>(A.med, x, c, g, H);
    double pu[D];
    if (D == 1) {
        const double nrm = fabs(ch[0]);
        const double r = fmax((ch[0] / nrm / c) * (ch[0] / nrm / c), 0.0);
        pu[0] = A.geo.inward * sqrt(r);
    } else {
        const double ta = fmax(fabs(tau), 1e-6);
        double t2 = 0.0;
        j = 0;
        for (int a = 0; a < D; ++a)
            if (a != na) {
                pu[a] = c * ch[1 + j] / ta;
                t2 += pu[a] * pu[a];
                ++j;
            }
        pu[na] = A.geo.inward * sqrt(fmax(1.0 - t2, 0.0));
    }
    double p[D];
    for (int a = 0; a < D; ++a) p[a] = 2.0 * pi * pu[a] / (D == 1 ? 1.0 : c);
    // spatial Hessian from the spacetime one (mT_inverse, tr_solver_utils.py:116-170)
    cd M[D][D];
    double np2 = 0.0;
    for (int a = 0; a < D; ++a) np2 += p[a] * p[a];
    const double npn = sqrt(np2);
    double xd[D], pd[D];
    for (int a = 0; a < D; ++a) {
        xd[a] = signum * c * p[a] / npn;
        pd[a] = -signum * g[a] * npn;
    }
    cd alpha[D];
    for (int a = 0; a < D; ++a) alpha[a] = cd{0.0, 2.0 * (pi * sig[a]) * (pi * sig[a]) / omega};
    cd num = alpha[0] + cd{pd[0] * xd[0], 0.0};
    for (int b = 1; b < D; ++b) {
        num = num + cd{-pd[b] * xd[b], 0.0} + (xd[b] * xd[b]) * alpha[b];
        const cd ur = cd{pd[b] / xd[0], 0.0} - (xd[b] / xd[0]) * alpha[b];
        M[0][b] = ur;
        M[b][0] = ur;
        for (int m = 1; m < D; ++m) M[b][m] = m == b ? alpha[b] : cd{0.0, 0.0};
    }
    M[0][0] = (1.0 / (xd[0] * xd[0])) * num;
    cd a = cd{ats * pc, ats * ps};
    bool placeholder = p[na] == 0.0;  // grazing: zero contribution, numerically safe values
    if (placeholder) a = cd{0.0, 0.0};
    if (A.b_inverse) {
        // -principal_b_inverse: i sign(W) / (2 c G), W = 2 pi tau,
        // G = sqrt(W^2 - c^2 |2 pi k_tan|^2); zero (and placeholders) when
        // evanescent, at W = 0 or within the relative guard of grazing.
        const double W = 2.0 * pi * tau;
        double q2 = 0.0;
        for (int b2 = 1; b2 < D; ++b2) q2 += (2.0 * pi * ch[b2]) * (2.0 * pi * ch[b2]);
        const double rad = W * W - (c * c) * q2;
        const double G = sqrt(fmax(rad, 0.0));
        const bool valid = rad > 0.0 && fabs(W) > 0.0 && G > A.guard * fabs(W);
        const double sw = W > 0.0 ? 1.0 : -1.0;
        a = valid ? a * cd{0.0, sw / (2.0 * c * G)} : cd{0.0, 0.0};
        placeholder |= !valid;
    }
    a = a * cd{A.values[i].x, A.values[i].y};
    if (placeholder) {
        for (int b2 = 0; b2 < D; ++b2) {
            p[b2] = 1.0;
            for (int m = 0; m < D; ++m) M[b2][m] = m == b2 ? cd{0.0, 1.0} : cd{0.0, 0.0};
        }
    }
    for (int b2 = 0; b2 < D; ++b2) {
        A.out.x[i * D + b2] = x[b2];
        A.out.p[i * D + b2] = p[b2];
        for (int m = 0; m < D; ++m) {
            A.out.M[2 * ((i * D + b2) * D + m)] = M[b2][m].re;
            A.out.M[2 * ((i * D + b2) * D + m) + 1] = M[b2][m].im;
        }
    }
    A.out.a[2 * i] = a.re;
    A.out.a[2 * i + 1] = a.im;
    A.out.omega[i] = omega;
    A.out.mode[i] = signum;
    A.out.t0[i] = t0;
}

struct ScatterArgs {
    const int64_t *idx;
    const double2 *g;
    int64_t n;
    double scale;
    int mask;
    int levels;
    int64_t ccum[9];
    double2 *G;
};

__global__ void scatter_kernel(ScatterArgs A) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= A.n) return;
    const int64_t f = A.idx[i];
    double m = A.scale;
    if (A.mask) {
        int l = 0;
        while (l < A.levels - 1 && f >= A.ccum[l + 1]) ++l;
        const int64_t seg = A.ccum[l + 1] - A.ccum[l];
        if (f - A.ccum[l] >= seg / 2) m = 0.0;
    }
    const double2 v = A.g[i];
    double2 o = A.G[f];
    A.G[f] = make_double2(o.x + m * v.x, o.y + m * v.y);
}

size_t a256(size_t x) { return (x + 255) & ~size_t(255); }

struct TopnLayout {
    size_t kin, kout, vin, vout, cub, total, cub_bytes;
};

TopnLayout topn_layout(int64_t total) {
    TopnLayout l{};
    cub::DeviceRadixSort::SortPairs(nullptr, l.cub_bytes, (const uint64_t *)nullptr, (uint64_t *)nullptr,
                                    (const int32_t *)nullptr, (int32_t *)nullptr, (int)total);
    size_t o = 0;
    l.kin = o; o = a256(o + 8 * total);
    l.kout = o; o = a256(o + 8 * total);
    l.vin = o; o = a256(o + 4 * total);
    l.vout = o; o = a256(o + 4 * total);
    l.cub = o; o = a256(o + l.cub_bytes);
    l.total = o;
    return l;
}

}  // namespace
}  // namespace msgb

using namespace msgb;

extern "C" size_t msgb_topn_workspace_size(int64_t total, int64_t n) {
    (void)n;
    if (total <= 0 || total > 0x7fffffffLL) return 0;
    return topn_layout(total).total;
}

extern "C" int msgb_topn(const double *keys, const double *coeffs, int64_t total, int64_t n, int64_t *idx,
                         double *values, void *workspace, size_t workspace_bytes, msgb_stream_t stream) {
    if (!keys || !idx) return fail(MSGB_ERR_ARG, "msgb_topn: NULL keys or idx");
    if (values && !coeffs) return fail(MSGB_ERR_ARG, "msgb_topn: values requested without coeffs");
    if (total <= 0 || total > 0x7fffffffLL) return fail(MSGB_ERR_UNSUPPORTED, "msgb_topn: total out of range");
    if (n <= 0) return fail(MSGB_ERR_ARG, "top_n threshold must be a positive integer.");
    if (n > total) n = total;
    const TopnLayout l = topn_layout(total);
    if (!workspace || workspace_bytes < l.total)
        return fail(MSGB_ERR_WORKSPACE, "msgb_topn: workspace too small: need %zu, got %zu", l.total, workspace_bytes);
    if (((uintptr_t)workspace & 255) != 0) return fail(MSGB_ERR_WORKSPACE, "workspace must be 256-byte aligned");
    cudaStream_t st = as_stream(stream);
    char *ws = (char *)workspace;
    uint64_t *kin = (uint64_t *)(ws + l.kin), *kout = (uint64_t *)(ws + l.kout);
    int32_t *vin = (int32_t *)(ws + l.vin), *vout = (int32_t *)(ws + l.vout);
    const unsigned blocks = (unsigned)((total + 255) / 256);
    key_bits_kernel<<<blocks, 256, 0, st>>>(keys, total, kin, vin);
    size_t cb = l.cub_bytes;
    cudaError_t e = cub::DeviceRadixSort::SortPairs(ws + l.cub, cb, kin, kout, vin, vout, (int)total, 0, 64, st);
    if (e != cudaSuccess) return fail(MSGB_ERR_CUDA, "msgb_topn sort: %s", cudaGetErrorString(e));
    take_last_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(vout, total, n, (const double2 *)coeffs, idx,
                                                                 (double2 *)values);
    return check_launch("msgb_topn");
}

extern "C" int msgb_beam_init(const msgb_mswpt *plan, const double *L, const int64_t *idx, const double *values,
                              int64_t n, const msgb_beam_out *out, msgb_stream_t stream) {
    if (!plan || !L || !out) return fail(MSGB_ERR_ARG, "msgb_beam_init: NULL argument");
    if (n == 0) return MSGB_OK;
    if (!idx || !out->x0 || !out->p0 || !out->alpha || !out->a0 || !out->omega)
        return fail(MSGB_ERR_ARG, "msgb_beam_init: NULL array");
    InitArgs A{};
    if (int e = plan_view(plan, A.v)) return e;
    for (int a = 0; a < 3; ++a) A.L[a] = a < A.v.nd ? L[a] : 1.0;
    A.idx = idx;
    A.values = (const double2 *)values;
    A.n = n;
    A.out = *out;
    beam_init_kernel<<<(unsigned)((n + 255) / 256), 256, 0, as_stream(stream)>>>(A);
    return check_launch("msgb_beam_init");
}

extern "C" int msgb_coefficients_dpdt(const msgb_mswpt *plan, const double *L, const msgb_medium *med,
                                      const double *a, const double *b, int branch, int apply_half_mask,
                                      double *out, double *keys, msgb_stream_t stream) {
    if (!plan || !L || !med || !a || !b || !out) return fail(MSGB_ERR_ARG, "msgb_coefficients_dpdt: NULL argument");
    if (branch != 1 && branch != -1) return fail(MSGB_ERR_ARG, "branch must be +1 or -1");
    DpdtArgs A{};
    if (int e = plan_view(plan, A.v)) return e;
    for (int i = 0; i < 3; ++i) A.L[i] = i < A.v.nd ? L[i] : 1.0;
    msgb_problem pr{};
    pr.ndim = A.v.nd;
    if (int e = medium_args(&pr, med, A.med)) return e;
    A.a = (const double2 *)a;
    A.b = (const double2 *)b;
    A.total = A.v.ccum[A.v.levels];
    A.branch = (double)branch;
    A.mask = apply_half_mask;
    A.out = (double2 *)out;
    A.keys = keys;
    if (A.total == 0) return MSGB_OK;
    const int blk = 256;
    const unsigned grid = (unsigned)((A.total + blk - 1) / blk);
    cudaStream_t st = as_stream(stream);
    switch (A.v.nd) {
        case 1: dpdt_kernel<1><<<grid, blk, 0, st>>>(A); break;
        case 2: dpdt_kernel<2><<<grid, blk, 0, st>>>(A); break;
        default: dpdt_kernel<3><<<grid, blk, 0, st>>>(A); break;
    }
    return check_launch("msgb_coefficients_dpdt");
}

extern "C" int msgb_tr_init(const msgb_mswpt *data_plan, const double *data_L, const msgb_tr_geometry *geo,
                            const msgb_medium *med, const int64_t *idx, const double *values, int64_t n,
                            int b_inverse, double relative_guard, const msgb_tr_beams *out,
                            msgb_stream_t stream) {
    if (!data_plan || !data_L || !geo || !med || !out) return fail(MSGB_ERR_ARG, "msgb_tr_init: NULL argument");
    if (n < 0) return fail(MSGB_ERR_ARG, "negative beam count");
    if (n == 0) return MSGB_OK;
    if (!idx || !values || !out->x || !out->p || !out->M || !out->a || !out->omega || !out->mode || !out->t0)
        return fail(MSGB_ERR_ARG, "msgb_tr_init: NULL array");
    TrInitArgs A{};
    if (int e = plan_view(data_plan, A.v)) return e;
    const int d = A.v.nd;
    if (geo->normal_axis < 0 || geo->normal_axis >= d) return fail(MSGB_ERR_ARG, "normal axis out of range");
    if (geo->inward != 1.0 && geo->inward != -1.0) return fail(MSGB_ERR_ARG, "inward must be +1 or -1");
    for (int a = 0; a < 3; ++a) A.L[a] = a < d ? data_L[a] : 1.0;
    A.geo = *geo;
    msgb_problem pr{};
    pr.ndim = d;
    if (int e = medium_args(&pr, med, A.med)) return e;
    A.idx = idx;
    A.values = (const double2 *)values;
    A.n = n;
    if (b_inverse && !(relative_guard >= 0.0 && relative_guard < 1.0))
        return fail(MSGB_ERR_ARG, "relative_guard must lie in [0, 1)");
    A.b_inverse = b_inverse != 0;
    A.guard = relative_guard;
    A.out = *out;
    const int blk = 128;
    const unsigned grid = (unsigned)((n + blk - 1) / blk);
    cudaStream_t st = as_stream(stream);
    switch (d) {
        case 1: tr_init_kernel<1><<<grid, blk, 0, st>>>(A); break;
        case 2: tr_init_kernel<2><<<grid, blk, 0, st>>>(A); break;
        default: tr_init_kernel<3><<<grid, blk, 0, st>>>(A); break;
    }
    return check_launch("msgb_tr_init");
}

extern "C" int msgb_scatter_coeff_grad(const int64_t *idx, const double *g, int64_t n, double scale,
                                       const msgb_mswpt *plan, int apply_half_mask, double *G,
                                       msgb_stream_t stream) {
    if (!idx || !g || !G) return fail(MSGB_ERR_ARG, "msgb_scatter_coeff_grad: NULL argument");
    if (n == 0) return MSGB_OK;
    ScatterArgs A{};
    A.idx = idx;
    A.g = (const double2 *)g;
    A.n = n;
    A.scale = scale;
    A.mask = apply_half_mask;
    A.G = (double2 *)G;
    if (apply_half_mask) {
        if (!plan) return fail(MSGB_ERR_ARG, "msgb_scatter_coeff_grad: half mask needs the plan");
        PlanView v;
        if (int e = plan_view(plan, v)) return e;
        A.levels = v.levels;
        for (int l = 0; l <= v.levels; ++l) A.ccum[l] = v.ccum[l];
    }
    scatter_kernel<<<(unsigned)((n + 255) / 256), 256, 0, as_stream(stream)>>>(A);
    return check_launch("msgb_scatter_coeff_grad");
}
