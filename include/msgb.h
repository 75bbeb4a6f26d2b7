/*
 * msgb.h - C ABI of libmsgb.so, the B200 (sm_100a) implementation of the
 * multiscale Gaussian beam (MSGB) forward operator and its exact transpose.
 *
 * Every entry point works on caller-owned device memory, is ordered on the
 * given CUDA stream, does not synchronise the host, and returns an int status
 * (MSGB_OK = 0).  msgb_last_error() returns a thread-local message for the
 * last failing call.  Entry points that need scratch memory take
 * (void* workspace, size_t workspace_bytes) and have a *_workspace_size query;
 * they never allocate.  Only msgb_mswpt_create allocates (the per-transform
 * device tables, once), and msgb_mswpt_destroy frees them.
 *
 * Reference interfaces replaced (paths relative to the beamax project root):
 *   MSWPT.forward / _compute_coeffs       beamax/transforms.py:591-733
 *   MSWPT.inverse                          beamax/transforms.py:735-850
 *   compute_coefficients (pos_only)        beamax/solvers/msgb_solvers/forward_solver_utils.py:716-786
 *   _threshold_top_n                       beamax/solvers/msgb_solvers/forward_solver_utils.py:65-89
 *   compute_forward_parameters             beamax/solvers/msgb_solvers/forward_solver_utils.py:255-373
 *   solve_hom_diag                         beamax/gb/gb_solvers.py:356-422
 *   compute_gaussian_beam_real (scan_real) beamax/gb/core.py:194-329
 *   compute_forward_result                 beamax/solvers/msgb_solvers/forward_solver_utils.py:652-713
 * The transpose entry points (msgb_adj_*, msgb_mswpt_adjoint) replace the
 * reference's jax.vjp of the forward (examples/diagnostics/msgb_adjoint_pairing.py:156-165).
 */
#ifndef MSGB_H
#define MSGB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st *msgb_stream_t; /* == cudaStream_t */

enum {
    MSGB_OK = 0,
    MSGB_ERR_ARG = 1,        /* invalid argument or shape */
    MSGB_ERR_WORKSPACE = 2,  /* workspace missing or too small */
    MSGB_ERR_CUDA = 3,       /* CUDA runtime / launch error */
    MSGB_ERR_UNSUPPORTED = 4,/* configuration outside what the kernels support */
    MSGB_ERR_NONFINITE = 5,  /* non-finite input detected */
    MSGB_ERR_TIMEOUT = 6     /* a bounded device wait ran out */
};

/* Domain, medium and acquisition grid (device pointers for ts / sensors). */
typedef struct msgb_problem {
    int32_t ndim;            /* 1, 2 or 3 */
    int32_t periodic[3];     /* per-axis periodic flags (geometry.py:25) */
    double L[3];             /* physical size per axis, N * dx (geometry.py:226-236) */
    double c;                /* constant sound speed (homogeneous entry points) */
    int64_t nt;              /* number of time samples */
    const double *ts;        /* (nt) */
    int64_t ns;              /* number of sensors */
    const double *sensors;   /* (ns, ndim), in the caller's order */
} msgb_problem;

/* Selected coefficients' beam data, positive branch (device, SoA).  Every
 * coefficient is propagated twice, with mode +1 and mode -1
 * (msgb_solver.py:612-619), so 2n beams are summed. */
typedef struct msgb_beam_set {
    int64_t n;
    const double *x0;        /* (n, ndim) initial centres */
    const double *p0;        /* (n, ndim) initial momenta, |p0| = 2 pi */
    const double *alpha;     /* (n, ndim) complex (re, im): diagonal of M0 */
    const double *a0;        /* (n) complex: amplitude; includes the coefficient for
                                the forward, the unit amplitude for the adjoint */
    const double *omega;     /* (n) frequency |xi| */
    int32_t modes;           /* which of the two branches are summed: 0 both (beam b < n
                                mode +1, b >= n mode -1, the real path's mirrored set),
                                1 only mode +1, 2 only mode -1 (the complex path's two
                                selections); homogeneous summations only */
} msgb_beam_set;

/* Optional sensor order for the FP32 summation (device pointers).  Tile i
 * holds the sorted sensors order[tile_offsets[i] .. tile_offsets[i+1]) (at
 * most 128); within a tile, groups of 16 consecutive sensors that lie on one
 * straight, evenly spaced run are evaluated with a complex-exponential
 * recurrence.  NULL: the library's own cell-Morton order. */
typedef struct msgb_sensor_tiling {
    int64_t n_tiles;
    const int32_t *order;         /* (ns) sorted position -> caller's sensor index */
    const int32_t *tile_offsets;  /* (n_tiles + 1) */
} msgb_sensor_tiling;

/* Options of the FP32 summation. */
typedef struct msgb_sum_opts {
    double cutoff;           /* skip a (beam, tile) pair when the Gaussian exponent
                                is provably above this many e-folds (<= 0: dense) */
    unsigned long long *eval_count; /* optional device counter: evaluated
                                (beam, t, sensor) triples are added to it */
    const msgb_sensor_tiling *tiling; /* optional (NULL) */
} msgb_sum_opts;

const char *msgb_last_error(void);
const char *msgb_version(void);

/* ---- Gaussian-beam summation: replaces compute_gaussian_beam_real with
 *      solve_hom_diag (gb/core.py:194-329, gb/gb_solvers.py:356-422) -------- */

/* Dense FP64 forward, reference semantics (no cutoff).
 * out: (nt, ns) FP64, overwritten. */
int msgb_sum_fwd_f64(const msgb_problem *prob, const msgb_beam_set *beams, double *out,
                     msgb_stream_t stream);

/* Exact transpose of msgb_sum_fwd_f64 down to the coefficients:
 * g[j] = sum_{mode, t, s} 2 data(t, s) conj(K_j(t, s)), contribution = 2 Re[c_j K_j].
 * beams->a0 must hold the unit amplitude.  data: (nt, ns) FP64.  g: (n) complex. */
int msgb_adj_gather_f64(const msgb_problem *prob, const msgb_beam_set *beams,
                        const double *data, double *g, msgb_stream_t stream);

/* FP32 forward with Kahan-compensated accumulation across beams, per-(beam,
 * time) FP64 range-reduced anchor phases and Gaussian cutoff culling.
 * out: (nt, ns) FP32.  The workspace (for n selected coefficients) covers
 * both this call and msgb_adj_gather_f32. */
size_t msgb_sum_f32_workspace_size(const msgb_problem *prob, int64_t n);
int msgb_sum_fwd_f32(const msgb_problem *prob, const msgb_beam_set *beams,
                     const msgb_sum_opts *opts, void *workspace, size_t workspace_bytes,
                     float *out, msgb_stream_t stream);

/* msgb_sum_fwd_f32 for callers that cannot allocate device memory: no
 * counterpart in the reference.  Meant for hosts that have no allocator to
 * give this library (an XLA custom call registered without a scratch buffer,
 * a runtime whose device memory is owned by another framework's pool, a
 * server that forbids allocation after start-up).  It calls no cudaMalloc,
 * cudaFree or allocating library routine; its scratch is a fixed array of
 * MSGB_SUM_F32_STATIC_SCRATCH_BYTES inside the library, resident on every GPU
 * that loads the library until the process exits.  Same inputs, output and
 * numerics as msgb_sum_fwd_f32 on the current device.
 *   - Limit: problems whose forward scratch exceeds the array are rejected
 *     with MSGB_ERR_UNSUPPORTED and a message giving the bytes needed (about
 *     44 B per coefficient plus 50-70 B per sensor: 65536 coefficients and
 *     2044 sensors take about 3 MB, and 16 MiB holds about 370000
 *     coefficients at that sensor count).
 *   - The first call on each device, with that device current, looks up the
 *     array's device address (cudaGetSymbolAddress); make that first call
 *     before any stream capture.  The stream must belong to the current
 *     device (checked: MSGB_ERR_ARG otherwise).
 *   - Every call shares the one array, which keeps the last call's contents
 *     (the call clears what must start at zero).  Calls whose executions
 *     overlap on the GPU (different streams, or concurrent host threads)
 *     race on it: order them on one stream or with events. */
#define MSGB_SUM_F32_STATIC_SCRATCH_BYTES (16u << 20)
int msgb_sum_fwd_f32_static(const msgb_problem *prob, const msgb_beam_set *beams,
                            const msgb_sum_opts *opts, float *out, msgb_stream_t stream);

/* FP32 transpose of msgb_sum_fwd_f32 (same culling), a deterministic
 * per-beam gather: work items are (time tile, range of beams); each item
 * sums its beams' conj(kernel) x data over every sensor tile and time of its
 * tile in a fixed order into one partial per (time tile, beam mode), and a
 * second kernel adds the partials over the time tiles in order.  No
 * floating-point atomics: results are bit-identical between runs.  data:
 * (nt, ns) FP32.  g: (n) complex FP64, overwritten.  The workspace holds the
 * partials (16 B per time tile of 32 samples and beam mode). */
int msgb_adj_gather_f32(const msgb_problem *prob, const msgb_beam_set *beams,
                        const msgb_sum_opts *opts, void *workspace, size_t workspace_bytes,
                        const float *data, double *g, msgb_stream_t stream);

/* ---- heterogeneous media: FP64 beam propagation ------------------------ */

#define MSGB_TIME_TILE 32          /* time samples per culling record */

enum {
    MSGB_MEDIUM_CONSTANT = 0,      /* c(x) = c */
    MSGB_MEDIUM_LINEAR = 1,        /* n-linear interpolation of grid values */
    MSGB_MEDIUM_BSPLINE3 = 2       /* cubic B-spline, coefficients prefiltered by the caller
                                      (scipy.ndimage.spline_filter, as utils/interp.py:66-73) */
};

/* Sound speed for the RK4 path (utils/interp.py:158-263): grid point k_a sits
 * at origin_a + k_a spacing_a; boundary 0 nearest (clamp), 1 wrap, 2 reflect,
 * 3 mirror (utils/interp.py:78-98). */
typedef struct msgb_medium {
    int32_t kind;
    int32_t boundary;
    int32_t n[3];
    double spacing[3];
    double origin[3];
    const double *coeffs;    /* device, prod(n) values (C order) */
    double c;                /* kind CONSTANT */
    double lam;              /* absorption lambda of coupled_rhs_absorption */
    const float *coeffs32;   /* optional: (coeffs - c_ref) in FP32, for msgb_ode_opts.medium_fp32 */
    double c_ref;
} msgb_medium;

/* Trajectory output for beams [b_first, b_first + nb) of the 2n beams (b >= n:
 * mode -1).  Any pointer may be NULL.  The amplitude is integrated from 1.
 *   rec64: (nt, nb) records of 2d + 2d^2 + 2 doubles: x, p, M (row-major,
 *          re/im interleaved), A (re, im).
 *   rec32: (nt, nb) records for the FP32 summation: x (d doubles, wrapped on
 *          periodic axes), w p (d doubles), w/2 Re M and w/2 Im M packed
 *          upper-triangular with doubled off-diagonals (d(d+1)/2 floats each),
 *          arg A and 2|A| (floats).
 *   cull:  (ceil(nt / MSGB_TIME_TILE), nb, 2d + 1) floats: bounding box of
 *          the centre over each time tile (lo, hi) and (w/2) min lambda_min(Im M).
 *   status: (nb) 0 ok, 1 non-finite state encountered, 2 max_steps reached
 *          (the adaptive integrator; the state then stays at its last value). */
typedef struct msgb_trajectories {
    int64_t nb;
    int64_t b_first;
    double *rec64;
    void *rec32;
    float *cull;
    int32_t *status;
    /* Compact FP32 store (used when rec32 is NULL and pool is not): records of
     * a (time tile, beam) pair are kept only when its culling box comes within
     * `live_cutoff` e-folds of at least one of the `n_boxes` sensor-tile boxes
     * (the summation's tiles, msgb_sum_f32_tile_boxes), in a block of
     * MSGB_TIME_TILE records taken from the pool.
     *   slot:      (ceil(nt / MSGB_TIME_TILE), nb) block index, -1 for a dead tile;
     *   pool:      (pool_blocks, MSGB_TIME_TILE) records in the rec32 layout;
     *   pool_cull: (pool_blocks, 2d + 1) the culling box of each block;
     *   pool_next: device counter of blocks taken (zeroed by the caller); a
     *              value above pool_blocks after the call means the pool ran
     *              out and the records are incomplete (integrate again with a
     *              larger pool or fewer beams).
     * Each lane of the integrator holds at most one block that no live tile
     * took, so pool_next ends at most (live tiles + lanes). */
    int32_t *slot;
    void *pool;
    float *pool_cull;
    int64_t pool_blocks;
    unsigned long long *pool_next;
    const float *live_boxes;       /* (n_boxes, 2d): lo then hi of each sensor tile */
    int64_t n_boxes;
    double live_cutoff;
} msgb_trajectories;

enum {
    MSGB_ODE_RK4 = 0,              /* fixed step: `substeps` equal steps per save interval */
    MSGB_ODE_DOPRI5 = 1            /* adaptive Dormand-Prince 5(4) */
};

/* Integrator settings; the adaptive fields mirror SolverConfig
 * (gb/gb_solvers.py:597-632: rtol 1e-7, atol 1e-9, max_steps 4096, dt0). */
typedef struct msgb_ode_opts {
    int32_t method;
    int32_t substeps;        /* RK4 */
    double rtol, atol;       /* DOPRI5: error norm RMS |e| / (atol + rtol max(|y0|, |y1|)) */
    double dt0;              /* DOPRI5 first step; <= 0 selects ts[1] - ts[0] */
    int64_t max_steps;       /* DOPRI5: accepted + rejected steps per beam (plus nt - 1
                                when steps end on the save times) */
    int32_t only_flagged;    /* nonzero: integrate only beams whose out->status entry is
                                nonzero (e.g. rejected surrogate predictions); the
                                records of the others are left as they are */
    int32_t dense_output;    /* DOPRI5 save times: 0 steps end on every save time (each
                                step at most one save interval); 1 steps follow the error
                                control and save times come from the continuous extension */
    unsigned long long *step_count; /* optional device counter (NULL: none): attempted
                                DOPRI5 steps (accepted + rejected) of the call are added to it */
    int32_t medium_fp32;     /* DOPRI5 with a grid medium and med->coeffs32, for the FP32 path:
                                evaluate c, grad c and hess c in FP32 (taps centred on the
                                nearest one, result + c_ref in FP64) and form the step-size
                                error norm in FP32.  Without dense_output the Hessian M and
                                the amplitude A are also integrated in FP32 (the ray x, p
                                stays FP64): the mixed-precision integrator, whose FP32
                                rounding stays far below the FP32 summation's.  0: every
                                operation in FP64 (the FP64 path). */
} msgb_ode_opts;

/* FP64 integration of coupled_rhs_absorption (gb/gb_solvers.py:787-867) for
 * each beam, state recorded at every ts; replaces solve_ODE_base
 * (gb/gb_solvers.py:940-1014, diffrax Tsit5 with PIDController and
 * SaveAt(ts)).  One thread per beam. */
int msgb_ode_trajectories(const msgb_problem *prob, const msgb_medium *med, const msgb_beam_set *beams,
                          const msgb_ode_opts *opts, const msgb_trajectories *out, msgb_stream_t stream);

/* msgb_ode_trajectories with method MSGB_ODE_RK4 and the given substeps. */
int msgb_rk4_trajectories(const msgb_problem *prob, const msgb_medium *med, const msgb_beam_set *beams,
                          int substeps, const msgb_trajectories *out, msgb_stream_t stream);

/* Summation from trajectories (beams [b_first, b_first + nb) of traj).  The
 * amplitude of beam b is a0[b mod n] times the trajectory's A.
 * FP64: dense, accumulates (+=) into out (nt, ns) FP64, which the caller
 * zeroes before the first chunk.
 * FP32: culled by the trajectory's boxes; Kahan state (2 nt ns floats) lives in
 * the workspace from the call with first_chunk != 0 to the call with
 * last_chunk != 0, which writes out (nt, ns) FP32.  All chunks of one
 * summation must use the same workspace and problem. */
int msgb_sum_fwd_f64_traj(const msgb_problem *prob, const msgb_beam_set *beams,
                          const msgb_trajectories *traj, double *out, msgb_stream_t stream);
int msgb_adj_gather_f64_traj(const msgb_problem *prob, const msgb_beam_set *beams,
                             const msgb_trajectories *traj, const double *data, double *g,
                             msgb_stream_t stream);
size_t msgb_sum_f32_traj_workspace_size(const msgb_problem *prob, int64_t nb_max);
int msgb_sum_fwd_f32_traj(const msgb_problem *prob, const msgb_beam_set *beams,
                          const msgb_trajectories *traj, const msgb_sum_opts *opts, int first_chunk,
                          int last_chunk, void *workspace, size_t workspace_bytes, float *out,
                          msgb_stream_t stream);
/* Number of sensor tiles of the FP32 summation for this problem and options
 * (opts->tiling's count, else one per 128 sensors), and their bounding boxes:
 * boxes (n_tiles, 2 ndim) floats, lo then hi, as the summation's culling uses
 * them.  The workspace is msgb_sum_f32_traj_workspace_size(prob, 0) bytes. */
int64_t msgb_sum_f32_tile_count(const msgb_problem *prob, const msgb_sum_opts *opts);
int msgb_sum_f32_tile_boxes(const msgb_problem *prob, const msgb_sum_opts *opts, void *workspace,
                            size_t workspace_bytes, float *boxes, msgb_stream_t stream);

/* g[b - b_first] for the chunk's beams (complex FP64, one entry per beam, not
 * per coefficient: the caller adds the two modes), deterministic as
 * msgb_adj_gather_f32; the workspace (sized for nb_max beams per chunk) holds
 * the partials. */
int msgb_adj_gather_f32_traj(const msgb_problem *prob, const msgb_beam_set *beams,
                             const msgb_trajectories *traj, const msgb_sum_opts *opts,
                             void *workspace, size_t workspace_bytes, const float *data, double *g,
                             msgb_stream_t stream);

/* ---- trajectory surrogate: data path around the MLP -------------------- */
/* No counterpart in the reference (it integrates every beam).  A BF16 MLP
 * predicts each beam's state as a correction to the homogeneous closed form
 * at c0 = c(x0); these entry points build its inputs and training targets
 * from trajectories and turn predictions back into msgb_trajectories records.
 * Rows are time-major: row q = kq * nb + (b - b_first). */
typedef struct msgb_surrogate_io {
    int64_t nb, b_first;       /* beams [b_first, b_first + nb) of the 2n */
    int64_t nq_t;              /* time samples per beam */
    const int32_t *t_index;    /* (nq_t) indices into ts, device; NULL: 0 .. nq_t - 1 */
    int32_t ld;                /* row stride of X / Y in elements */
} msgb_surrogate_io;

/* Acceptance of predicted trajectories.  A beam is accepted when
 * max_t |c(x)|p| / (c0 |p0|) - 1| <= residual_tol (status 3 otherwise) and
 * w |p0| pos_err <= phase_tol (status 4 otherwise), pos_err being the
 * surrogate's validated position error in metres. */
typedef struct msgb_surrogate_accept {
    double residual_tol;
    double phase_tol;
    double pos_err;
} msgb_surrogate_accept;

/* X (rows, ld) BF16 features: x0 / L, mode p0 / |p0|, log10 w - 3,
 * log10 Im alpha + 3, (t - ts[0]) / (ts[nt-1] - ts[0]); 3d + 2 columns, the
 * rest zero. */
int msgb_surrogate_features(const msgb_problem *prob, const msgb_medium *med, const msgb_beam_set *beams,
                            const msgb_surrogate_io *io, uint16_t *X, msgb_stream_t stream);
/* Y (rows, ld) FP32 targets from rec64 (nt, nb, 2d + 2d^2 + 2) of the same
 * chunk: (x - x_hom) / (c0 T), (p - p0) / |p0|, (M^-1 - M_hom^-1) |p0| / (c0 T)
 * (upper triangle, real parts then imaginary parts), log(A / A_hom) (re, im):
 * 6, 12 or 20 columns for d = 1, 2, 3. */
int msgb_surrogate_targets(const msgb_problem *prob, const msgb_medium *med, const msgb_beam_set *beams,
                           const msgb_surrogate_io *io, const double *rec64, float *Y,
                           msgb_stream_t stream);
/* Records from standardised predictions Y (every time, t_index NULL):
 * y * stdv + mean per column, then the inverse of the target map.  Writes
 * the records of beams [io->b_first, io->b_first + io->nb), which must lie in
 * out's chunk, and their out->status entries (0 accepted, 3 or 4 rejected). */
int msgb_surrogate_records(const msgb_problem *prob, const msgb_medium *med, const msgb_beam_set *beams,
                           const msgb_surrogate_io *io, const float *Y, const float *mean,
                           const float *stdv, const msgb_surrogate_accept *accept,
                           const msgb_trajectories *out, msgb_stream_t stream);

/* ---- tensor-core BF16 GEMM and MLP kernels (trajectory surrogate) ------ */

/* C = A B^T (+ bias) on the tcgen05 tensor cores, FP32 accumulation in tensor
 * memory.  A (M x K) and B (N x K) are BF16 with element strides (sAm, sAk)
 * and (sBn, sBk); N is a multiple of 16 in [16, 256].  C32 receives the FP32
 * pre-activation, C16 the BF16 activation (act 0: identity, 1: SiLU). */
typedef struct msgb_gemm {
    const void *A;
    int64_t sAm, sAk;
    const void *B;
    int64_t sBn, sBk;
    int32_t M, N, K;
    const float *bias;
    int32_t act;
    float *C32;
    int64_t ldc32;
    void *C16;
    int64_t ldc16;
    int *error_flag;  /* device int, set to 1 if a tensor-core wait ran out; may be NULL */
} msgb_gemm;

int msgb_gemm_bf16(const msgb_gemm *p, msgb_stream_t stream);
/* dZ = dA * silu'(Z) elementwise (FP32 in; FP32 and/or BF16 out). */
int msgb_silu_backward(const float *dA, const float *Z, int64_t n, float *dZ32, void *dZ16,
                       msgb_stream_t stream);
/* out[n] = sum_m X[m, n], fixed order. */
int msgb_colsum(const float *X, int M, int N, int64_t ld, float *out, msgb_stream_t stream);
/* Adam step (FP32 master weights, optional BF16 copy). */
int msgb_adam(float *w, const float *g, float *m1, float *m2, int64_t n, double lr, double b1, double b2,
              double eps, int64_t step, void *w16, msgb_stream_t stream);
int msgb_to_bf16(const float *x, int64_t n, void *y, msgb_stream_t stream);

/* ---- MSWPT tiling (transforms.py:357-850) ------------------------------ */

typedef struct msgb_mswpt msgb_mswpt;

/* Host-side description of a transform (all pointers are host memory). */
typedef struct msgb_mswpt_desc {
    int32_t ndim;
    int32_t N[3];
    int32_t aspect[3];           /* box_aspect_ratio */
    int32_t redundancy;          /* 1 or 2 */
    int32_t num_levels;
    int32_t total_boxes;
    const int32_t *box_length;   /* (num_levels) box_lengths (smallest axis) */
    const int32_t *box_level;    /* (total_boxes) level of every box */
    const int32_t *centres;      /* (total_boxes, ndim) centres_ndim */
    const int32_t *box_shape;    /* (num_levels, ndim) half supports (box_shapes) */
    const int64_t *coeffs_cumsum;/* (num_levels + 1) */
    const int32_t *boxes_cumsum; /* (num_levels + 1) */
    const double *gfilt;         /* concatenated per-level packed g, C order */
    const int64_t *gfilt_offset; /* (num_levels) offsets into gfilt */
    const double *sum_gsquare;   /* (prod N) */
    /* lattice lookup used by the deterministic synthesis gather:
     * per level, outer box counts per axis and a table mapping the lattice
     * multi-index (C order) to the global box id or -1 (cut out). */
    const int32_t *lattice_counts;  /* (num_levels, ndim) */
    const int32_t *lattice_first;   /* (num_levels, ndim) first lattice centre per axis */
    const int32_t *lattice_step;    /* (num_levels, ndim) lattice step per axis */
    const int64_t *lattice_offset;  /* (num_levels) offsets into lattice_box */
    const int32_t *lattice_box;     /* concatenated tables */
} msgb_mswpt_desc;

int msgb_mswpt_create(const msgb_mswpt_desc *desc, msgb_mswpt **plan);
int msgb_mswpt_destroy(msgb_mswpt *plan);
int64_t msgb_mswpt_total_coeffs(const msgb_mswpt *plan);
size_t msgb_mswpt_workspace_size(const msgb_mswpt *plan);

/* Analysis: coeffs = scale * MSWPT.forward(in) [* half_mask].
 * in: prod(N) values, FP64, real (is_complex = 0) or interleaved complex.
 * coeffs: (total_coeffs) complex FP64.  With keys != NULL also writes the
 * top_n selection key sqrt(re*re + im*im) of every output coefficient. */
int msgb_mswpt_forward(const msgb_mswpt *plan, const double *in, int is_complex,
                       int input_is_fourier, double scale, int apply_half_mask,
                       double *coeffs, double *keys, void *workspace, size_t workspace_bytes,
                       msgb_stream_t stream);

/* Synthesis.  mode bit 0 clear: MSWPT.inverse (transforms.py:735-850); set:
 * the Hermitian adjoint of msgb_mswpt_forward (spatial input).  mode bit 1
 * set: return the (shifted, unitary) Fourier-domain field instead of the
 * spatial one.  out: prod(N) values, FP64; the real part only when
 * real_output != 0, else interleaved complex.  The coefficient buffer is
 * not modified. */
int msgb_mswpt_synthesis(const msgb_mswpt *plan, const double *coeffs, int mode,
                         int real_output, double *out, void *workspace,
                         size_t workspace_bytes, msgb_stream_t stream);

/* ---- top_n selection (forward_solver_utils.py:65-89) ------------------- */

/* Selects the n largest keys; ties at the threshold keep the highest indices
 * (jnp.argpartition semantics); emits them ordered by (key, index) ascending.
 * idx: (n) int64; values: (n) complex gathered from coeffs. */
size_t msgb_topn_workspace_size(int64_t total, int64_t n);
int msgb_topn(const double *keys, const double *coeffs, int64_t total, int64_t n,
              int64_t *idx, double *values, void *workspace, size_t workspace_bytes,
              msgb_stream_t stream);

/* The other thresholds of threshold_coefficients (forward_solver_utils.py:
 * 14-178, 181-230) over the same keys |c| and coefficients:
 *   hard           |c| > val
 *   percentile     |c| > jnp.percentile(|c|, val) ("linear")
 *   hard_reassign  |c| >= val max|c|, values scaled by sqrt(sum|c|^2 / sum kept |c|^2)
 *   bao_energy     |c| |centre of the coefficient's box|^d > val (needs plan)
 *   perc_max_abs   |c| > val max|c|
 * Writes the selected flat indices in ascending order to idx[0 .. *count),
 * their (scaled) coefficients to values, and the count to *count (device). */
enum {
    MSGB_THR_HARD = 0,
    MSGB_THR_PERCENTILE = 1,
    MSGB_THR_HARD_REASSIGN = 2,
    MSGB_THR_BAO_ENERGY = 3,
    MSGB_THR_PERC_MAX_ABS = 4
};
size_t msgb_threshold_workspace_size(int64_t total);
int msgb_threshold(int strategy, double val, const double *keys, const double *coeffs, int64_t total,
                   const msgb_mswpt *plan, int64_t *idx, double *values, int64_t *count,
                   void *workspace, size_t workspace_bytes, msgb_stream_t stream);

/* ---- beam initialisation (forward_solver_utils.py:255-373) ------------- */

typedef struct msgb_beam_out {
    double *x0, *p0, *alpha, *a0, *omega;  /* layouts as in msgb_beam_set */
    double *a0_unit;                        /* (n) complex, optional (NULL) */
} msgb_beam_out;

/* Beam data for n selected flat indices; values (complex, may be NULL) are
 * multiplied into a0.  L: physical domain size per axis. */
int msgb_beam_init(const msgb_mswpt *plan, const double *L, const int64_t *idx,
                   const double *values, int64_t n, const msgb_beam_out *out,
                   msgb_stream_t stream);

/* compute_coefficients with a non-zero initial time derivative
 * (forward_solver_utils.py:716-786): from a = MSWPT(p0) and b = MSWPT(dpdt)
 * (complex, unscaled), out = 0.5 (a + branch i b / vg) with
 * vg = c(x_b) |2 pi centre / L| per coefficient (gb_utils.py:11-44; x_b the
 * coefficient's position, c from the medium), branch +1 (c_pos) or -1
 * (c_neg); with apply_half_mask the second half of every level is zeroed.
 * keys (optional): |out| for the selection.  L: host array of ndim lengths. */
int msgb_coefficients_dpdt(const msgb_mswpt *plan, const double *L, const msgb_medium *med,
                           const double *a, const double *b, int branch, int apply_half_mask,
                           double *out, double *keys, msgb_stream_t stream);

/* ---- time reversal ------------------------------------------------------ */
/* MSGBSolver.time_reversal (solvers/msgb_solvers/msgb_solver.py:984-1111):
 * beams launched from a planar detector at their data time
 * (tr_solver_utils.py:205-440), integrated back to t = 0 and summed at image
 * points with msgb_sum_fwd_f64_traj (one time, rec64 of the final states,
 * beam amplitudes a, frequencies omega). */
typedef struct msgb_tr_geometry {
    int32_t normal_axis;     /* spatial axis normal to the detector plane */
    double normal_value;     /* the detector's coordinate on that axis */
    double inward;           /* +1 or -1: sign of the normal momentum into the domain */
} msgb_tr_geometry;

typedef struct msgb_tr_beams {
    int64_t n;
    double *x, *p;           /* (n, d) position and momentum on the detector */
    double *M;               /* (n, d, d) complex spatial Hessian */
    double *a;               /* (n) complex amplitude, times the coefficient */
    double *omega;           /* (n) frequency |tau| */
    double *mode;            /* (n) branch -sign(tau) */
    double *t0;              /* (n) launch time */
} msgb_tr_beams;

/* compute_TR_parameters (tr_solver_utils.py:205-440) for the selected
 * data-transform coefficients (flat indices idx, values c[idx]): data_plan is
 * the boundary-data MSWPT (axis 0 time, then the detector's tangential axes),
 * data_L its physical lengths (host, ndim), med the medium at the detector.
 * With b_inverse != 0, compute_adj_parameters (adjoint_solver_utils.py:
 * 78-200) instead: the amplitude times -B^{-1}(tau, k_tan, c(x_T)) of
 * principal_b_inverse (:17-75) with the given relative_guard, and beams whose
 * multiplier is 0 get the grazing placeholders.  Writes every field of out. */
int msgb_tr_init(const msgb_mswpt *data_plan, const double *data_L, const msgb_tr_geometry *geo,
                 const msgb_medium *med, const int64_t *idx, const double *values, int64_t n,
                 int b_inverse, double relative_guard, const msgb_tr_beams *out, msgb_stream_t stream);

/* _form_adjoint_source (msgb_solver.py:68-120): out (nt, ns) = -c_s^2
 * Re(ifft_t(2 pi i fftfreq(nt, dt) fft_t(window r))), r (nt, ns) row-major,
 * window NULL, (nt) (window_is_time_only) or (nt, ns), c_at_sources (ns).
 * Creates (and destroys) a batched cuFFT plan per call; the workspace holds
 * the spectrum and cuFFT's work area. */
size_t msgb_adjoint_source_workspace_size(int64_t nt, int64_t ns);
int msgb_adjoint_source(const double *data, const double *window, int window_is_time_only, int64_t nt,
                        int64_t ns, double dt, const double *c_at_sources, double *out, void *workspace,
                        size_t workspace_bytes, msgb_stream_t stream);

/* c(x) of the medium at n points x (n, ndim) (Domain.c_fn, geometry.py:
 * 176-221, for the medium kinds of msgb_medium). */
int msgb_medium_speed(int32_t ndim, const msgb_medium *med, const double *x, int64_t n, double *c,
                      msgb_stream_t stream);

/* Each beam integrated from its launch time back to t = 0 (adaptive FP64,
 * opts as msgb_ode_trajectories; time reversed by flipping the branch and the
 * absorption sign), amplitude from 1.  rec64: (n, 2d + 2d^2 + 2) final states;
 * status (n): 0 ok, 1 non-finite, 2 step budget exhausted.  prob supplies
 * ndim, L and periodic. */
int msgb_tr_final_states(const msgb_problem *prob, const msgb_medium *med, const msgb_tr_beams *beams,
                         const msgb_ode_opts *opts, double *rec64, int32_t *status, msgb_stream_t stream);

/* ---- adjoint scatter to coefficient space ------------------------------ */

/* G[idx[j]] += scale * g[j]; G must be zeroed by the caller.  Complex FP64.
 * Precondition: the n indices are distinct (a selection of top_n or of a
 * threshold always is).  Each entry is updated by one thread without atomics,
 * so duplicate indices race and leave G undefined at those entries. */
int msgb_scatter_coeff_grad(const int64_t *idx, const double *g, int64_t n, double scale,
                            const msgb_mswpt *plan, int apply_half_mask, double *G,
                            msgb_stream_t stream);

/* ---- throughput probes (measurement; no counterpart in the reference) ---
 * The roofline denominators of the FP32 summation, the beam ODE (FP32 and FP64) and the
 * special-function unit, measured on the device that runs them: blocks x
 * threads threads each run 8 independent chains of `iters` operations of one
 * kind.  The caller times the launch on its stream and divides
 * msgb_peak_probe_ops() (flops, FMA = 2; MUFU: operations) by the time.
 * sink: (blocks * threads) floats, overwritten. */
enum {
    MSGB_PEAK_FP32 = 0,      /* scalar FFMA */
    MSGB_PEAK_FP32X2 = 1,    /* paired FFMA2 (two FP32 lanes per instruction) */
    MSGB_PEAK_FP64 = 2,      /* DFMA */
    MSGB_PEAK_MUFU = 3       /* sin.approx (MUFU) */
};
double msgb_peak_probe_ops(int kind, int64_t iters, int blocks, int threads);
int msgb_peak_probe(int kind, int64_t iters, int blocks, int threads, float *sink, msgb_stream_t stream);

#ifdef __cplusplus
}
#endif
#endif /* MSGB_H */
