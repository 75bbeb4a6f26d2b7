// Coefficient thresholds other than top_n: hard, percentile, hard_reassign,
// bao_energy and perc_max_abs (forward_solver_utils.py:14-178, dispatched by
// threshold_coefficients :181-230).  Every strategy is a mask over the
// half-masked positive-branch coefficients, compacted into ascending flat
// indices (the order jnp.nonzero returns).  Thresholds that depend on the
// data (the maximum, the percentile, the energy ratio) are computed on the
// device, so a selection costs one device-to-host read of the count.
//
// Magnitudes are the selection keys |c| = sqrt(re*re + im*im) that
// msgb_mswpt_forward writes.  percentile follows jnp.percentile's "linear"
// rule: with s the ascending magnitudes and q = val / 100 * (total - 1),
// s[floor q] * (1 - f) + s[floor q + 1] * f, f = q - floor q.  The padded
// entries (-1 index, value 0) that percentile and perc_max_abs return in
// the reference describe zero-amplitude beams and are not produced here.
#include <cub/cub.cuh>

#include "common.cuh"

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

struct Scalars {
    double max_abs;     // max |c|
    double thresh;      // comparison threshold on |c| (or |c| nx for bao_energy)
    double ratio;       // hard_reassign energy ratio, 1 otherwise
    double energy_all;  // sum |c|^2
    double energy_kept; // sum |c|^2 over the kept coefficients (hard_reassign)
};

struct BaoArgs {
    int nd, levels;
    int64_t ccum[9];
    int bcum[9];
    int64_t per_box[8];
    const int32_t *centres;
};

__device__ double bao_weight(const BaoArgs &b, int64_t i) {
    int l = 0;
    while (l + 1 < b.levels && i >= b.ccum[l + 1]) ++l;
    const int64_t box = b.bcum[l] + (i - b.ccum[l]) / b.per_box[l];
    double n2 = 0.0;
    for (int a = 0; a < b.nd; ++a) {
        const double c = (double)b.centres[box * b.nd + a];
        n2 += c * c;
    }
    const double r = sqrt(n2);
    double w = 1.0;
    for (int a = 0; a < b.nd; ++a) w *= r;
    return w;
}

struct Keep {
    int strategy;
    double val;
    const double *keys;
    const Scalars *s;
    BaoArgs bao;
    __device__ bool operator()(int64_t i) const {
        const double k = keys[i];
        switch (strategy) {
            case MSGB_THR_HARD: return k > val;
            case MSGB_THR_PERCENTILE:
            case MSGB_THR_PERC_MAX_ABS: return k > s->thresh;
            case MSGB_THR_HARD_REASSIGN:
                return s->max_abs > 0.0 && k >= s->thresh && s->ratio > 0.0 && k * s->ratio > 0.0;
            default: return k * bao_weight(bao, i) > val;
        }
    }
};

struct Square {
    __device__ double operator()(double k) const { return k * k; }
};
struct KeptSquare {
    const double *keys;
    const Scalars *s;
    __device__ double operator()(int64_t i) const {
        const double k = keys[i];
        return (s->max_abs > 0.0 && k >= s->thresh) ? k * k : 0.0;
    }
};

__global__ void key_bits64(const double *keys, int64_t n, uint64_t *kb) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) {
        double k = keys[i];
        if (k == 0.0) k = 0.0;
        kb[i] = (uint64_t)__double_as_longlong(k);
    }
}

__global__ void percentile_kernel(const uint64_t *sorted, int64_t n, double val, Scalars *s) {
    const double q = val / 100.0 * (double)(n - 1);
    double lo = floor(q);
    if (lo < 0.0) lo = 0.0;
    if (lo > (double)(n - 1)) lo = (double)(n - 1);
    const int64_t il = (int64_t)lo, ih = il + 1 < n ? il + 1 : n - 1;
    const double f = q - lo;
    const double a = __longlong_as_double((long long)sorted[il]), b = __longlong_as_double((long long)sorted[ih]);
    s->thresh = a * (1.0 - f) + b * f;
    s->ratio = 1.0;
}

__global__ void max_based_kernel(int strategy, double val, Scalars *s) {
    s->thresh = s->max_abs * val;
    s->ratio = 1.0;
    (void)strategy;
}

__global__ void ratio_kernel(Scalars *s) {
    const double re = s->energy_kept, te = s->energy_all;
    s->ratio = re > 0.0 ? sqrt(te / re) : 0.0;
}

__global__ void set_unit_kernel(Scalars *s) { s->ratio = 1.0; }

__global__ void gather_kernel(const int64_t *idx, const int64_t *count, const double2 *coeffs, const Scalars *s,
                              double2 *values) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= *count) return;
    const double2 c = coeffs[idx[i]];
    const double r = s->ratio;
    values[i] = make_double2(c.x * r, c.y * r);
}

struct ThrLayout {
    size_t kb, kbs, scal, cub, total, cub_bytes;
};

size_t a256(size_t x) { return (x + 255) & ~size_t(255); }

ThrLayout thr_layout(int64_t total) {
    ThrLayout l{};
    size_t b1 = 0, b2 = 0, b3 = 0, b4 = 0;
    cub::DeviceRadixSort::SortKeys(nullptr, b1, (const uint64_t *)nullptr, (uint64_t *)nullptr, (int)total);
    cub::DeviceReduce::Max(nullptr, b2, (const double *)nullptr, (double *)nullptr, (int)total);
    cub::CountingInputIterator<int64_t> it(0);
    Keep keep{};
    cub::DeviceSelect::If(nullptr, b3, it, (int64_t *)nullptr, (int64_t *)nullptr, (int)total, keep);
    cub::TransformInputIterator<double, Square, const double *> sq((const double *)nullptr, Square{});
    cub::DeviceReduce::Sum(nullptr, b4, sq, (double *)nullptr, (int)total);
    l.cub_bytes = b1 > b2 ? b1 : b2;
    if (b3 > l.cub_bytes) l.cub_bytes = b3;
    if (b4 > l.cub_bytes) l.cub_bytes = b4;
    size_t o = 0;
    l.kb = o; o = a256(o + 8 * total);
    l.kbs = o; o = a256(o + 8 * total);
    l.scal = o; o = a256(o + sizeof(Scalars));
    l.cub = o; o = a256(o + l.cub_bytes);
    l.total = o;
    return l;
}

}  // namespace
}  // namespace msgb

using namespace msgb;

extern "C" size_t msgb_threshold_workspace_size(int64_t total) {
    if (total <= 0 || total > 0x7fffffffLL) return 0;
    return thr_layout(total).total;
}

extern "C" int msgb_threshold(int strategy, double val, const double *keys, const double *coeffs, int64_t total,
                              const msgb_mswpt *plan, int64_t *idx, double *values, int64_t *count, void *workspace,
                              size_t workspace_bytes, msgb_stream_t stream) {
    if (!keys || !coeffs || !idx || !values || !count) return fail(MSGB_ERR_ARG, "msgb_threshold: NULL argument");
    if (total <= 0 || total > 0x7fffffffLL) return fail(MSGB_ERR_UNSUPPORTED, "msgb_threshold: total out of range");
    if (strategy < MSGB_THR_HARD || strategy > MSGB_THR_PERC_MAX_ABS)
        return fail(MSGB_ERR_ARG, "Invalid thresholding strategy: %d", strategy);
    if (!isfinite(val)) return fail(MSGB_ERR_ARG, "threshold must be finite");
    if (strategy == MSGB_THR_PERCENTILE && !(val >= 0.0 && val <= 100.0))
        return fail(MSGB_ERR_ARG, "percentile threshold must lie in [0, 100].");
    if ((strategy == MSGB_THR_HARD_REASSIGN || strategy == MSGB_THR_PERC_MAX_ABS) && !(val >= 0.0 && val <= 1.0))
        return fail(MSGB_ERR_ARG, "threshold must lie in [0, 1].");
    BaoArgs bao{};
    if (strategy == MSGB_THR_BAO_ENERGY) {
        if (!plan) return fail(MSGB_ERR_ARG, "bao_energy thresholding requires wpt.");
        PlanView v;
        if (int e = plan_view(plan, v)) return e;
        if (v.ccum[v.levels] != total) return fail(MSGB_ERR_ARG, "coefficient count differs from the MSWPT plan");
        bao.nd = v.nd;
        bao.levels = v.levels;
        bao.centres = v.centres;
        for (int l = 0; l <= v.levels; ++l) {
            bao.ccum[l] = v.ccum[l];
            bao.bcum[l] = v.bcum[l];
        }
        for (int l = 0; l < v.levels; ++l) {
            int64_t pb = 1;
            for (int a = 0; a < v.nd; ++a) pb *= 2 * v.bshape[l][a];  // support = twice the half support
            bao.per_box[l] = pb;
        }
    }
    const ThrLayout l = thr_layout(total);
    if (!workspace || workspace_bytes < l.total)
        return fail(MSGB_ERR_WORKSPACE, "msgb_threshold: workspace too small: need %zu, got %zu", l.total,
                    workspace_bytes);
    if (((uintptr_t)workspace & 255) != 0) return fail(MSGB_ERR_WORKSPACE, "workspace must be 256-byte aligned");
    cudaStream_t st = as_stream(stream);
    char *ws = (char *)workspace;
    Scalars *s = (Scalars *)(ws + l.scal);
    void *cubws = ws + l.cub;
    const int blk = 256;
    const unsigned grid = (unsigned)((total + blk - 1) / blk);
    cudaError_t e = cudaSuccess;
    size_t cb = l.cub_bytes;
    if (strategy == MSGB_THR_PERCENTILE) {
        uint64_t *kb = (uint64_t *)(ws + l.kb), *kbs = (uint64_t *)(ws + l.kbs);
        key_bits64<<<grid, blk, 0, st>>>(keys, total, kb);
        e = cub::DeviceRadixSort::SortKeys(cubws, cb, kb, kbs, (int)total, 0, 64, st);
        if (e == cudaSuccess) percentile_kernel<<<1, 1, 0, st>>>(kbs, total, val, s);
    } else if (strategy == MSGB_THR_PERC_MAX_ABS || strategy == MSGB_THR_HARD_REASSIGN) {
        e = cub::DeviceReduce::Max(cubws, cb, keys, &s->max_abs, (int)total, st);
        if (e == cudaSuccess) max_based_kernel<<<1, 1, 0, st>>>(strategy, val, s);
        if (e == cudaSuccess && strategy == MSGB_THR_HARD_REASSIGN) {
            cub::TransformInputIterator<double, Square, const double *> sq(keys, Square{});
            cb = l.cub_bytes;
            e = cub::DeviceReduce::Sum(cubws, cb, sq, &s->energy_all, (int)total, st);
            if (e == cudaSuccess) {
                cub::CountingInputIterator<int64_t> it(0);
                cub::TransformInputIterator<double, KeptSquare, cub::CountingInputIterator<int64_t>> kq(
                    it, KeptSquare{keys, s});
                cb = l.cub_bytes;
                e = cub::DeviceReduce::Sum(cubws, cb, kq, &s->energy_kept, (int)total, st);
            }
            if (e == cudaSuccess) ratio_kernel<<<1, 1, 0, st>>>(s);
        }
    } else {
        set_unit_kernel<<<1, 1, 0, st>>>(s);
    }
    if (e != cudaSuccess) return fail(MSGB_ERR_CUDA, "msgb_threshold: %s", cudaGetErrorString(e));
    Keep keep{strategy, val, keys, s, bao};
    cub::CountingInputIterator<int64_t> it(0);
    cb = l.cub_bytes;
    e = cub::DeviceSelect::If(cubws, cb, it, idx, count, (int)total, keep, st);
    if (e != cudaSuccess) return fail(MSGB_ERR_CUDA, "msgb_threshold: %s", cudaGetErrorString(e));
    gather_kernel<<<grid, blk, 0, st>>>(idx, count, (const double2 *)coeffs, s, (double2 *)values);
    return check_launch("msgb_threshold");
}
