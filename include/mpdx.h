/*
 * libmpdataxx_b200 -- C ABI of the B200 (sm_100a) MPDATA / pressure-solve backend.
 *
 * This is the boundary that a concurr::cuda backend (header-only C++, see
 * libmpdataxx_b200/include/libmpdata++/concurr/cuda.hpp) or any FFI binds.
 * Plain pointers and sizes only.  Each entry point names the reference
 * interface it replaces (paths inside the libmpdata++ source tree).
 *
 * Fields live on the device for the life of the handle.  Host buffers are
 * caller-owned and copied synchronously; element strides describe the host
 * layout (so the reference's 3D storage order -- k fastest, then i, then j,
 * libmpdata++/blitz.hpp:116-117 -- is accepted as is).
 *
 * Threading: a handle is used from one host thread at a time; its work is
 * serialised on the handle's CUDA stream.
 */
#ifndef MPDX_H
#define MPDX_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes; the C++ header maps each to the reference's exception text. */
typedef enum {
  MPDX_OK = 0,
  MPDX_E_GRID = 1,        /* "libmpdata++: bogus grid size" (solver_common.hpp:246-248) */
  MPDX_E_DIVERGENT = 2,   /* "libmpdata++: initial advector field is divergent" (solver_2d.hpp:290-291) */
  MPDX_E_PRS_STUCK = 3,   /* "libmpdata++: stuck in pressure solver" (mpdata_rhs_vip_prs_common.hpp:121-125) */
  MPDX_E_UNSUPPORTED = 4, /* option / boundary-condition combination not built on this backend */
  MPDX_E_CUDA = 5,        /* CUDA runtime error (message in mpdx_last_error) */
  MPDX_E_TIMEOUT = 6,     /* a bounded device-side wait gave up */
  MPDX_E_ARG = 7          /* invalid argument (null pointer, index out of range, ...) */
} mpdx_status;

/* boundary kinds (libmpdata++/bcond/detail/bcond_common.hpp bcond_e).  GNDSKY is the
 * 3D ground / sky condition of bcond/gndsky_3d.hpp: the rigid condition on every
 * field this backend fills (its own fills are for subgrid-scale fields only). */
enum { MPDX_BC_CYCLIC = 0, MPDX_BC_OPEN = 1, MPDX_BC_RIGID = 2, MPDX_BC_GNDSKY = 3 };

/* velocity absorber (ct_params_t::vip_vab, mpdata_rhs_vip_common.hpp:16-21) */
enum { MPDX_VAB_NONE = 0, MPDX_VAB_EXPL = 1, MPDX_VAB_IMPL = 2 };

/* solver families (solvers::mpdata, solvers::boussinesq) */
enum { MPDX_SOLVER_MPDATA = 0, MPDX_SOLVER_BOUSSINESQ = 1 };

/* pressure schemes (solvers::prs_scheme_t, mpdata_rhs_vip_prs.hpp:17-30) */
enum { MPDX_PRS_CR = 0, MPDX_PRS_GCRK = 1 };

/* preconditioner inside GCR: identity (the reference's) or the learned one */
enum { MPDX_PRECOND_IDENTITY = 0, MPDX_PRECOND_LEARNED = 1 };

/* execution path: AUTO picks the fused kernels when the configuration allows
 * (all-cyclic, supported opts, periodic seams consistent) else GENERAL, which
 * runs one kernel per reference formula; both are CUDA. */
enum { MPDX_PATH_AUTO = 0, MPDX_PATH_GENERAL = 1, MPDX_PATH_FUSED = 2 };

/* field kinds for mpdx_set_field / mpdx_get_field */
enum {
  MPDX_FIELD_ADVECTEE = 0,   /* idx = equation; interior n0 x n1 x n2 */
  MPDX_FIELD_ADVECTOR = 1,   /* idx = dimension; reference view extents (below) */
  MPDX_FIELD_SCLR_ARRAY = 2, /* idx = MPDX_SCLR_* named scalar array */
  MPDX_FIELD_PRESSURE = 3,   /* Boussinesq: Phi, interior */
  MPDX_FIELD_G = 4           /* g_factor() with the nug option: G, interior (sharedmem.hpp:373-380) */
};
/* scalar arrays: sclr_array("tht_e"), ("tht_abs"), ("hflux_frc") (boussinesq_common.hpp:20-60),
 * vab_coefficient() and vab_relaxed_state(d) (concurr_common.hpp:415-433) as MPDX_SCLR_VAB_RELAX + d */
enum { MPDX_SCLR_THT_E = 0, MPDX_SCLR_THT_ABS = 1, MPDX_SCLR_HFLUX_FRC = 2, MPDX_SCLR_VAB_COEFF = 3,
       MPDX_SCLR_VAB_RELAX = 4 };

/* Run-time and compile-time parameters of one solver (ct_params_t + rt_params_t,
 * libmpdata++/opts.hpp:81-100, solver_common.hpp:217-221, mpdata_common.hpp:74-78,
 * mpdata_rhs_vip_prs_common.hpp:193-196, boussinesq_common.hpp:32-35). */
typedef struct {
  int solver;              /* MPDX_SOLVER_* */
  int n_dims;              /* 1..3 */
  int n_eqns;              /* advected equations */
  int grid[3];             /* grid_size */
  uint64_t opts;           /* opts bitmask, same bit values as libmpdata++/opts.hpp */
  int n_iters;             /* MPDATA iterations (default 2) */
  int dtype;               /* sizeof(real_t): 4 (float) or 8 (double) */
  int bcs[6];              /* MPDX_BC_* for (x left, x right, y left, y right, z left, z right) */
  double dt, di, dj, dk;   /* time step and grid spacings */
  double max_abs_div_eps;  /* < 0 selects the reference default, machine epsilon of real_t */
  int path;                /* MPDX_PATH_* */
  /* Boussinesq / pressure solve */
  int prs_scheme;          /* MPDX_PRS_CR or MPDX_PRS_GCRK */
  int prs_k_iters;         /* k of GCR(k) for MPDX_PRS_GCRK (default 4) */
  double prs_tol;          /* stop when max|err| <= prs_tol / dt */
  double g, tht_ref;       /* gravity, reference potential temperature */
  int ix_u, ix_v, ix_w, ix_tht;  /* equation indices (ct_params_t::ix); ix_v = -1 in 2D */
  int precond;             /* MPDX_PRECOND_* */
  int prs_fp64;            /* 1: pressure fields in FP64 even when real_t is float */
  int upwind_filter_freq;  /* rt_params upwind_filter_freq (mpdata_common.hpp:77): every n-th step is upwind only; 0 = never */
  int impl_tht;            /* ct_params_t::impl_tht: theta is the perturbation from tht_e, its coupling with w implicit (boussinesq_impl.hpp) */
  int vip_vab;             /* ct_params_t::vip_vab: MPDX_VAB_* velocity absorber */
  int sptl_intrp;          /* ct_params_t::sptl_intrp (formulae_mpdata_common.hpp:21-26) of the div_3rd spatial
                              terms: 0 exact, 1 aver2, 2 aver4 */
} mpdx_config;

typedef struct mpdx_solver *mpdx_handle;

/* Per-step device-side statistics, read back on demand. */
typedef struct {
  int64_t timestep;
  double time;
  double mass;             /* FP64 compensated sum of advectee(0) over the interior */
  double min, max;         /* of advectee(0) */
  int64_t gcr_iters;       /* iterations of the last pressure solve (Boussinesq) */
  int64_t gcr_iters_total; /* since creation */
  double gcr_residual;     /* max|err| at the end of the last pressure solve */
  int path;                /* path used by the last advance (MPDX_PATH_GENERAL/FUSED) */
  double gcr_ms;           /* device time of the last pressure solve, start to max|err| <= prs_tol / dt */
  int gcr_fallback;        /* 1 if the last solve left the learned preconditioner for plain GCR,
                              2 if it was redone from its start with plain GCR alone */
} mpdx_step_stats;

/* Fill *cfg with the reference defaults (opts = iga|fct, n_iters = 2, ...). */
void mpdx_config_default(mpdx_config *cfg);

/* concurr::<backend><solver_t, bc...> run(p)  (concurr_common.hpp:176-187, any.hpp:15-74):
 * allocates every device field of the solver. */
mpdx_status mpdx_create(const mpdx_config *cfg, mpdx_handle *out);

/* run.advectee(e) = ... / run.advector(d) = ... / run.sclr_array(name) = ...
 * (concurr_common.hpp:387-433, sharedmem.hpp:411-456, 543-577).
 * Advector views follow the reference: lower bound (-1, 0, 0); extents
 * (n0, n1, n2) for d = 0 and (n0 + 1, n1, n2) for d >= 1.  Strides are in
 * elements of real_t; NULL strides mean C order. */
mpdx_status mpdx_set_field(mpdx_handle h, int kind, int idx, const void *host, const int64_t *strides);
mpdx_status mpdx_get_field(mpdx_handle h, int kind, int idx, void *host, const int64_t *strides);

/* Same with device pointers (C order), for callers that keep data on the GPU.
 * The copy is ordered after all work already issued to the legacy default
 * stream (where a producer that uses no streams of its own writes the buffer);
 * a buffer written on any other stream must be complete (synchronised by the
 * caller) before the call.  Both calls return after the copy. */
mpdx_status mpdx_set_field_device(mpdx_handle h, int kind, int idx, const void *dev);
mpdx_status mpdx_get_field_device(mpdx_handle h, int kind, int idx, void *dev);

/* Asynchronous transfers for pipelined host loops (no counterpart in the reference):
 * `host` must be page-locked (pinned) and C-ordered, and must stay valid and
 * unchanged until mpdx_sync(h) returns.  Uploads and downloads run on two
 * transfer streams of the handle, each after all compute enqueued before the
 * call and after the previous asynchronous transfer of the same field; later
 * compute (mpdx_advance) and the synchronous entry points wait for them.  An
 * upload of the advector can therefore overlap the download of the previous
 * step's advectee. */
mpdx_status mpdx_set_field_async(mpdx_handle h, int kind, int idx, const void *host);
mpdx_status mpdx_get_field_async(mpdx_handle h, int kind, int idx, void *host);

/* run.advance(nt)  (concurr_common.hpp:380-385 -> solver_common.hpp:270-358).
 * Asynchronous with respect to the host except on the first call (the
 * divergence check of hook_ante_loop reads one device scalar back). */
mpdx_status mpdx_advance(mpdx_handle h, int64_t nt);

/* Blocks until the handle's stream and its transfer streams are idle. */
mpdx_status mpdx_sync(mpdx_handle h);

/* run.min()/max()/timestep plus FP64 mass and pressure-solver counters
 * (sharedmem.hpp:115-246). */
mpdx_status mpdx_stats(mpdx_handle h, mpdx_step_stats *out);

/* The handle's CUDA stream (cudaStream_t), for callers that order work with it. */
void *mpdx_stream(mpdx_handle h);

/* Plane copies of the fused FP32 3D kernel (all boundaries cyclic, iga or
 * iga|fct, n_iters 2), process-wide: mode 1 (the default) copies each plane of
 * a CTA whose tile lies inside the periods along the two inner axes with one
 * bulk-tensor copy (TMA) counted on an mbarrier, mode 0 copies with per-thread
 * asynchronous copies everywhere; both give bitwise-identical results.  A
 * negative mode only queries.  Returns the mode before the call.  A bulk copy
 * whose completion wait gives up (after about two seconds) makes the next call
 * on any handle fail with MPDX_E_CUDA. */
int mpdx_fused3d_bulk_copies(int mode);

/* Planes per CTA of the fused 3D kernel (the length of the x-chunk one CTA
 * marches through), process-wide: 0 (the default) lets each handle tune it on
 * its first fused steps, a positive value fixes it (a multiple of 4 from 8 to
 * 512); a negative value only queries.  Returns the setting before the call, or
 * -1 for an invalid value (which changes nothing).  Every value gives
 * bitwise-identical fields: a point is computed by the same operations whichever
 * CTA holds it.  No reference counterpart (the reference's threads split the
 * domain along x by its own rule, concurr/detail/concurr_common.hpp). */
int mpdx_fused3d_planes_per_cta(int lx);

/* The tuner of a handle that takes the fused 3D path: its first fused step runs
 * untimed with 64 planes per CTA, then each candidate in lx[] (24, 32, 40, 48,
 * 64, 80, 96 and 128 planes) runs two timed steps (each waiting for its own end
 * on the host, so a caller that captures mpdx_advance into a CUDA graph does so
 * after these 17 steps, or fixes the value with mpdx_fused3d_planes_per_cta), then the
 * fastest is kept for the handle's life.  chosen is 0 while tuning (or on a
 * handle that has not taken the fused 3D path); ms[] holds each candidate's time
 * per step once the choice is made. */
typedef struct {
  int chosen;
  int n_candidates;
  int lx[8];
  float ms[8];
} mpdx_tuning3d;
mpdx_status mpdx_fused3d_tuning(mpdx_handle h, mpdx_tuning3d *out);

/* Message of the last failing call on this handle ("" if none). */
const char *mpdx_last_error(mpdx_handle h);

/* Message of the last failing mpdx_create in this thread. */
const char *mpdx_create_error(void);

void mpdx_destroy(mpdx_handle h);

/* FP64 compensated sum over [0,m0) x [0,m1) x [0,m2), minimum and maximum over
 * [0,n0) x [0,n1) x [0,n2) of a caller-owned device array (dtype 4 or 8,
 * element strides), written as three doubles to the device buffer dev_out,
 * asynchronously on `stream` (a cudaStream_t; NULL for the legacy stream).
 *
 * No counterpart in the reference.  It allocates nothing: for callers that
 * cannot allocate device memory where they need these numbers (device memory
 * owned by a caching or pooled allocator, fixed memory budgets).  Its scratch
 * is one fixed-size array in device memory: at most 8192 points along axis 0
 * (larger extents return MPDX_E_ARG with the reason in err).  The first call
 * on a device looks up that array's address and should come before any stream
 * capture; calls on one device that overlap on the GPU race on the array. */
mpdx_status mpdx_field_stats_noalloc(const void *dev_field, int dtype, const int64_t *n, const int64_t *strides,
                                     const int64_t *m, double *dev_out, void *stream, char *err, int errlen);

/* ---- Batched advance of independent 2D problems ----
 *
 * No counterpart in the reference, where every run object advances alone.  A
 * batch groups existing handles (2D, same dtype, opts and n_iters, one
 * equation, cyclic boundaries, opts within fct/iga) and advances all of them
 * together: MPDX_BATCH_PERSISTENT runs one persistent fused launch per step,
 * whose tile shape an autotuner picks by timing the first steps (results do
 * not depend on it), captured with the next steps in a CUDA graph;
 * MPDX_BATCH_PER_PROBLEM launches the fused kernel once per problem per step.
 * The handles stay usable (fields, stats) between batched advances; the batch
 * must be destroyed before its handles.  Errors of mpdx_batch_create are in
 * mpdx_create_error(). */
typedef struct mpdx_batch *mpdx_batch_handle;
enum { MPDX_BATCH_PERSISTENT = 0, MPDX_BATCH_PER_PROBLEM = 1 };

typedef struct {
  int n_problems;
  int64_t cells;        /* sum over the problems of n0 x n1 */
  int mode;             /* MPDX_BATCH_* */
  int tile_nt, tile_lx; /* tile chosen by the autotuner (0 until tuning ends) */
  int grid;             /* CTAs of the persistent launch chosen by the autotuner */
  int n_candidates;     /* candidates timed by the autotuner: rows per item 16, 32, 64, 128 with
                           every resident CTA, then the same with half of them */
  double tune_ms[8];    /* mean ms of a batched step per candidate, over 3 steps (0 = not measured yet) */
} mpdx_batch_info;

mpdx_status mpdx_batch_create(const mpdx_handle *handles, int n, int mode, mpdx_batch_handle *out);
mpdx_status mpdx_batch_advance(mpdx_batch_handle b, int64_t nt);
mpdx_status mpdx_batch_get_info(mpdx_batch_handle b, mpdx_batch_info *out);
mpdx_status mpdx_batch_sync(mpdx_batch_handle b);
const char *mpdx_batch_last_error(mpdx_batch_handle b);
void mpdx_batch_destroy(mpdx_batch_handle b);

/* ---- Learned preconditioner inside a Boussinesq solver's GCR ----
 *
 * No counterpart in the reference (its cr / gcrk solvers use no
 * preconditioner).  FP64 pressure solves only (dtype 8, or prs_fp64).
 * mpdx_precond_record keeps (residual, correction Phi_end - Phi) pairs of the
 * next pressure solves on the device (the start and iterations 16, 32, 64 of
 * each, up to max_pairs); mpdx_precond_train runs `steps` Adam steps (linear
 * warm-up, cosine decay to 1 % of lr) on the energy loss of
 * mpdx_precond_loss_grad over randomly drawn pairs, the last fifth of the pairs
 * (at most 8) held out, and keeps the weights with the lowest held-out loss seen (never
 * worse than the weights it started from); *final_loss is that held-out loss
 * (1 = no correction).  With mpdx_precond_enable every pressure solve starts
 * with nl learned corrections, Phi += beta q along q = net(err) with the step
 * beta = -<err, q> / <q, lap q> that minimises the error in the operator's energy
 * norm (the training norm), and continues with plain GCR from the iterate they
 * reach.  nl = 1 unless mpdx_precond_set_directions sets another count (0..64)
 * or -1, which chooses nl in {1, 2, 4, 0} by the measured device times of
 * earlier solves (each tried twice, then the fastest, one re-measured every 64
 * solves; a choice by single solves, which does not see that the learned
 * corrections also make the next solves start closer to their solution).
 * The stopping test (max|err| <= prs_tol / dt) is unchanged: only the iteration
 * count and time change.  mpdx_precond_directions gives the nl of the last
 * learned solve (-1 before the first).  Weights are exchanged in the mpdx_pcnet
 * layout. */
mpdx_status mpdx_precond_record(mpdx_handle h, int64_t max_pairs);
mpdx_status mpdx_precond_train(mpdx_handle h, int64_t steps, double lr, uint64_t seed, double *final_loss);
mpdx_status mpdx_precond_enable(mpdx_handle h, int on);
mpdx_status mpdx_precond_set_directions(mpdx_handle h, int64_t nl);
int64_t mpdx_precond_directions(mpdx_handle h);
int64_t mpdx_precond_pairs(mpdx_handle h);
int64_t mpdx_precond_num_params(mpdx_handle h);
mpdx_status mpdx_precond_get_params(mpdx_handle h, float *host);
mpdx_status mpdx_precond_set_params(mpdx_handle h, const float *host);
/* The training loss for one pair given by the caller (no counterpart in the
 * reference): residual r and correction t (interior, C order, FP64 on the host;
 * A t = -r for the solve's operator A), network output q = net(r) scaled by c:
 * *loss = sum_d |G_d e| ^2 / sum_d |G_d t|^2 with e = c q - t and G_d the pressure
 * solve's centred gradient along axis d (pressure halo rules, zero on a rigid
 * wall): the error's energy, which for cyclic axes is e^T (-A) e, and which with
 * rigid walls (where -A is not symmetric and its quadratic form can be negative)
 * stays non-negative; 1 for a zero output.  Its gradient with respect to the
 * network parameters goes into grad (host, mpdx_precond_num_params floats; NULL
 * for the loss alone). */
mpdx_status mpdx_precond_loss_grad(mpdx_handle h, const double *r, const double *t, double c, double *loss, float *grad);

/* ---- Learned GCR preconditioner network on its own ----
 *
 * No counterpart in the reference.  A linear 4-level 3D (or 2D) U-net that maps
 * a residual field to a search direction, with BF16 tensor-core convolutions
 * (architecture in libmpdataxx_b200/csrc/precond.cu).  grid: points per axis;
 * wrap[d] = 1 pads axis d cyclically, 0 with zeros; channels: the four levels'
 * channel counts (8, 16, 32 or 64; level 0 at most 16).  Parameters are FP32
 * in the order e0 e1 e2 e3 m3 d2 d1 d0 q, each weight (cout, taps, cin) followed
 * by its bias (cout); taps run over offsets -1..1 with the last axis fastest.
 * Host arrays are C-ordered over the grid.  Errors of create are in
 * mpdx_pcnet_create_error(). */
typedef struct mpdx_pcnet *mpdx_pcnet_handle;
mpdx_status mpdx_pcnet_create(int nd, const int *grid, const int *wrap, const int *channels, uint64_t seed,
                              mpdx_pcnet_handle *out);
const char *mpdx_pcnet_create_error(void);
int64_t mpdx_pcnet_num_params(mpdx_pcnet_handle h);
mpdx_status mpdx_pcnet_set_params(mpdx_pcnet_handle h, const float *host);
mpdx_status mpdx_pcnet_get_params(mpdx_pcnet_handle h, float *host);
/* q = net(r) */
mpdx_status mpdx_pcnet_forward(mpdx_pcnet_handle h, const float *r_host, float *q_host);
/* gradient of sum(dq * net(r)) with respect to every parameter */
mpdx_status mpdx_pcnet_backward(mpdx_pcnet_handle h, const float *r_host, const float *dq_host, float *grad_host);
/* one Adam step (weights only; the biases stay as they are) on mean((net(r) - target)^2) */
mpdx_status mpdx_pcnet_train_step(mpdx_pcnet_handle h, const float *r_host, const float *target_host, float lr,
                                  double *loss);
const char *mpdx_pcnet_last_error(mpdx_pcnet_handle h);
void mpdx_pcnet_destroy(mpdx_pcnet_handle h);

#ifdef __cplusplus
}
#endif

#endif /* MPDX_H */
