// C ABI plumbing: thread-local error messages, argument validation and the
// conversion of public descriptors to kernel arguments.
#include <cstdarg>
#include <cstring>

#include "common.cuh"

namespace msgb {

static thread_local char g_err[1024] = "";

void set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

int fail(int code, const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

int check_launch(const char *what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(MSGB_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
    return MSGB_OK;
}

int validate_problem(const msgb_problem *p) {
    if (!p) return fail(MSGB_ERR_ARG, "problem descriptor is NULL");
    if (p->ndim < 1 || p->ndim > 3) return fail(MSGB_ERR_ARG, "ndim must be 1, 2 or 3 (got %d)", p->ndim);
    if (p->nt < 0 || p->ns < 0) return fail(MSGB_ERR_ARG, "negative nt or ns");
    if (p->nt > 0 && !p->ts) return fail(MSGB_ERR_ARG, "ts is NULL");
    if (p->ns > 0 && !p->sensors) return fail(MSGB_ERR_ARG, "sensors is NULL");
    if (!(p->c > 0.0) || !std::isfinite(p->c)) return fail(MSGB_ERR_ARG, "sound speed must be finite and > 0");
    for (int i = 0; i < p->ndim; ++i)
        if (!(p->L[i] > 0.0) || !std::isfinite(p->L[i])) return fail(MSGB_ERR_ARG, "domain size must be finite and > 0");
    return MSGB_OK;
}

int validate_beams(const msgb_problem *p, const msgb_beam_set *b) {
    (void)p;
    if (!b) return fail(MSGB_ERR_ARG, "beam set is NULL");
    if (b->n < 0) return fail(MSGB_ERR_ARG, "negative beam count");
    if (b->n > 0 && (!b->x0 || !b->p0 || !b->alpha || !b->a0 || !b->omega))
        return fail(MSGB_ERR_ARG, "beam arrays must not be NULL");
    if (b->modes < 0 || b->modes > 2) return fail(MSGB_ERR_ARG, "beam modes must be 0, 1 or 2");
    return MSGB_OK;
}

ProbArgs to_args(const msgb_problem *p) {
    ProbArgs a{};
    a.nd = p->ndim;
    for (int i = 0; i < 3; ++i) {
        a.periodic[i] = i < p->ndim ? (p->periodic[i] != 0) : 0;
        a.L[i] = i < p->ndim ? p->L[i] : 1.0;
    }
    a.c = p->c;
    a.nt = p->nt;
    a.ns = p->ns;
    a.ts = p->ts;
    a.sensors = p->sensors;
    return a;
}

BeamArgs to_args(const msgb_beam_set *b) {
    BeamArgs a{};
    a.n = b->n;
    a.x0 = b->x0;
    a.p0 = b->p0;
    a.alpha = b->alpha;
    a.a0 = b->a0;
    a.omega = b->omega;
    a.modes = b->modes;
    return a;
}

}  // namespace msgb

extern "C" const char *msgb_last_error(void) { return msgb::g_err; }
extern "C" const char *msgb_version(void) { return "libmsgb 0.1 sm_100a"; }
