/*
 * uniphot_b200 -- C ABI of the B200-native per-island VarPro-LM forced
 * photometry solve.
 *
 * The reference (uniphot / tract7dt) exposes this path as Python functions
 * over JAX device arrays; this ABI is the boundary a maintainer binds with
 * ctypes (the Python package's _lib module is such a binding).  Every entry point returns an int status
 * (UPH_OK on success) and never throws; uph_last_error() gives the text of
 * the last failure on a context.  All pointers are plain host pointers unless
 * the name says _device; sizes are element counts.
 *
 * Reference interfaces replaced (paths relative to the reference project):
 *   uph_upload_field        <- island_stage._shard_setup device upload of the
 *                              padded field stacks (fit/grid_gpu/island_stage.py:146-240)
 *                              and island_fit's pad+upload (island_solver.py:3334-3344)
 *   uph_upload_psf_poly     <- build_psf_tree (island_solver.py:1851-1871)
 *   uph_upload_psf_mog      <- (no reference counterpart: the analytic PSF of
 *                              the north-star render mode)
 *   uph_upload_sersic_table <- sersic_mog.get_table_jax (sersic_mog.py:59-78)
 *   uph_subtract_tile_backgrounds <- the padded field stacks' frozen per-tile
 *                              background subtraction (island_stage.py:1728-1751)
 *   uph_scene_subtract_stars <- the field-wide star scene subtraction
 *                              (island_stage.py:2024-2118, _star_stamps_jit :99-130)
 *   uph_upload_exp_mog      <- source_model.EXP_AMP / EXP_VAR (source_model.py:
 *                              56-75), the "direct" backend's mixture
 *   uph_run_chunk           <- run_class_chunk (island_solver.py:2793-3131)
 *                              for the legacy/clip/proposals step protocol
 */
#ifndef UNIPHOT_B200_H
#define UNIPHOT_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define UPH_OK 0
#define UPH_ERR_INVALID 1   /* bad argument / unsupported option            */
#define UPH_ERR_OOM 2       /* device allocation failed (caller may halve)  */
#define UPH_ERR_CUDA 3      /* any other CUDA runtime error                  */
#define UPH_ERR_TIMEOUT 4   /* a bounded device wait gave up                 */
#define UPH_ERR_STATE 5     /* call order violated (e.g. no field uploaded)  */

#define UPH_RENDER_REFERENCE 0  /* pixelised polynomial PSF, Lanczos-3 shift */
#define UPH_RENDER_ANALYTIC 1   /* Gaussian-mixture PSF (analytic convolution) */

typedef struct uph_ctx uph_ctx;

/* One solver class: (bbox B, nsrc N, stamp tier T) plus solver knobs.
 * Mirrors make_class_kernels(plan, n_bands, n_terms, ...)
 * (island_solver.py:1874-1922). */
typedef struct uph_class_desc {
  int32_t bbox;             /* B: island window side (pixels)              */
  int32_t nsrc;             /* N: member slots per island                  */
  int32_t tier;             /* T: odd stamp side                           */
  int32_t render_mode;      /* UPH_RENDER_*                                */
  float reg;                /* flux-solve ridge on real members (1e-9)     */
  float pos_step_max;       /* per-step position clip (0.5 px)             */
  float chi2_ftol_rel;      /* relative dchi2 convergence prong (1e-4)     */
  float step_tol_pix;       /* position step prong (0.1 px)                */
  int32_t un_freeze_steps;  /* u_n annealing budget (0 = never)            */
  int32_t has_priors;       /* nonlinear Gaussian priors present           */
  int32_t native_stamp;     /* odd native PSF stamp side: a star's model is
                               zero outside it (the reference zero-pads its
                               native PSF to the tier); 0 = tier            */
  int32_t precision;        /* UPH_PRECISION_PLAIN: FP32 Gram on CUDA cores;
                               UPH_PRECISION_MIXED: islands with more than
                               tc_min_rows Gram rows form it on the tensor
                               cores from BF16 hi/lo pairs with FP32
                               accumulation, in residual form             */
  int32_t tc_min_rows;      /* mixed form: Gram-row threshold of the
                               tensor-core path; < 0 selects the default
                               (UPH_TC_MIN_ROWS_DEFAULT)                   */
  int32_t stall_changed;    /* stall_count_mode: 0 "proposals" (legacy);
                               1 "changed": a reject counts toward the stall
                               only when its proposal differs from the
                               previous rejected one; identical-proposal
                               runs set the diverged flag in the loop
                               (island_solver.py:1118-1208)                */
  int32_t convergence_dlnp; /* 1: convergence "dlnp" (island_solver.py:
                               1210-1333): chi2 carried in float64,
                               absolute sub-quantum prongs, reject-exits
                               at the lam cap or on a no-move proposal,
                               plateau-certified exits reported converged;
                               implies the "changed" stall counting        */
  float plateau_dlnp_tol;   /* dlnp: the quantum is 2 * this (0.5)         */
  int32_t bg_joint;         /* 1: each band's planar background (1, X, Y
                               over the island window) is solved with the
                               fluxes in the inner linear step; 0: the data
                               are background-subtracted (the reference's
                               island mode)                                */
  float tc_cond_max;        /* mixed form: islands whose members' scaled
                               normal matrix has a conditioning indicator
                               above this (in any band) form the Gram in
                               FP32; < 0 selects UPH_TC_COND_MAX_DEFAULT  */
  int32_t step_tr;          /* step_mode: 0 "clip" (damped step, per-
                               parameter clips, lam x10 / x0.1); 1
                               "trust_region" (island_solver.py:1004-1116):
                               scaled dogleg inside a radius carried in the
                               lam slot (0 = unset, seeded by the first
                               Gauss-Newton step), radius updated from the
                               chi2 gain ratio; excludes stall_changed and
                               convergence_dlnp                            */
  int32_t param_errors;     /* 1: after the loop, the marginal covariance of
                               the nonlinear parameters at the final
                               parameters (island_solver.py:1484-1547):
                               the undamped Gauss-Newton matrix relinearised
                               there, static keep mask, plus the prior
                               diagonal, inverted in float64; returned in
                               uph_chunk_out.perr                          */
  int32_t flux_marg;        /* 1: the shape-marginalised flux-variance
                               increment (island_solver.py:1549-1613):
                               per band and extended member, J Sigma J^T
                               with J the flux solution's sensitivity to
                               the extended members' kept parameters and
                               Sigma the covariance of param_errors (which
                               this pass runs too); uph_chunk_out.femarg  */
  int32_t source_metrics;   /* 1: per-member model-quality metrics at the
                               final fit (island_solver.py:1639-1715):
                               rchisq, fracflux, fracin, fracmasked and the
                               per-band window flux; uph_chunk_out.smetrics
                               and .swin                                   */
  int32_t re_profile;       /* 1: chi2 profile along each extended member's
                               log-radius at the final fit, at the offsets
                               UPH_REPROF_DELTAS (island_solver.py:1779-
                               1792); uph_chunk_out.reprof                 */
  int32_t residual;         /* 1: band-coadded residual sum_b w (d - model)
                               and weight sum_b w over the island window
                               at the final fit (island_solver.py:1615-
                               1637); uph_chunk_out.resid and .resid_w     */
  int32_t scene_subtract;   /* 1: the field stacks are scene-subtracted; each
                               island's window gets its members added back
                               at their seed parameters and S1 fluxes,
                               sum_k member_s1_flux[k, b] m_k(seed)
                               (island_solver.py:1795-1818, 2781-2790), in
                               a private copy of the window, before the
                               solve; needs uph_chunk_in.member_s1_flux   */
  int32_t render_direct;    /* reference render mode: EXP galaxies by the
                               legacy "direct" backend (source_model.py:
                               218-256, 298-303): the exponential mixture
                               of uph_upload_exp_mog at pixel centres, unit
                               sum, convolved ("same") with the PSF stamp
                               and renormalised to unit sum, in float64;
                               position partials through the PSF's spatial
                               variation, shape partials by float64 central
                               differences (step 1e-6).  STAR and EXP
                               members only; tiers up to UPH_DIRECT_MAX_T */
} uph_class_desc;

#define UPH_DIRECT_MAX_T 111

/* log-radius offsets of the Re profile (the reference's REPROF_DELTAS_LN,
 * island_plan.py:58-60) */
#define UPH_REPROF_K 12
#define UPH_REPROF_DELTAS {-2.5f, -1.5f, -0.9f, -0.5f, -0.25f, -0.1f, \
                           0.1f, 0.25f, 0.5f, 0.9f, 1.5f, 2.5f}

#define UPH_TC_MIN_ROWS_DEFAULT 24
#define UPH_TC_COND_MAX_DEFAULT 10.0f

#define UPH_PRECISION_PLAIN 0
#define UPH_PRECISION_MIXED 1

/* Per-island inputs of one chunk of n islands (class_host_arrays rows;
 * island_plan.py:493-700).  Shapes: [n], [n*N], [n*N*6]. */
typedef struct uph_chunk_in {
  int32_t n_islands;
  const int32_t* ox;          /* [n]   window origin in the padded stack   */
  const int32_t* oy;          /* [n]                                        */
  const float* x0b;           /* [n]   window origin in field coords        */
  const float* y0b;           /* [n]                                        */
  const int32_t* stype;       /* [n*N] SOURCE_STAR=0, EXP=1, DEV=2, SERSIC=3 */
  const float* n_frozen;      /* [n*N] Sersic n when u_n is not free        */
  const uint8_t* free_n;      /* [n*N]                                      */
  const uint8_t* mmask;       /* [n*N] real member slot                     */
  const uint8_t* keep;        /* [n*N*6] fitted parameter mask              */
  const float* p0;            /* [n*N*6] (x, y, logre, ee1, ee2, u_n)       */
  const float* lower;         /* [n*N*6] box bounds                         */
  const float* upper;         /* [n*N*6]                                    */
  const float* prior_mean;    /* [n*N*6]                                    */
  const float* prior_inv_sigma; /* [n*N*6] 0 = no prior                     */
  /* optional LM carry state (NULL = fresh start from p0):
   * run_class_chunk(init_state=...) keys p, lam, chi2, consec, nrej, nst */
  const float* init_lam;      /* [n]                                        */
  const float* init_chi2;     /* [n]                                        */
  const int32_t* init_consec; /* [n]                                        */
  const int32_t* init_nrej;   /* [n]                                        */
  const int32_t* init_nst;    /* [n]                                        */
  /* optional "changed"-mode tracker carry (NULL = zeros):                   */
  const int32_t* init_n_same; /* [n]     identical-proposal reject run      */
  const float* init_prej;     /* [n*N*6] last rejected proposal             */
  const uint8_t* init_diverged; /* [n]   sticky diverged flag               */
  /* scene subtract (uph_class_desc.scene_subtract):                          */
  const float* member_s1_flux;  /* [n*N*nb] members' S1 fluxes (0 for the
                                   members not subtracted field-wide)      */
  const float* seed_p;          /* [n*N*6] seed parameters of the add-back;
                                   NULL = p0                               */
} uph_chunk_in;

/* Per-island outputs (run_class_chunk's dict).  Shapes as noted. */
typedef struct uph_chunk_out {
  float* p;             /* [n*N*6]                                         */
  float* fluxes;        /* [n*nb*N]  per-band VarPro fluxes                */
  float* ferr;          /* [n*nb*N]  sqrt(diag inv A64)                    */
  float* chi2;          /* [n]                                             */
  uint8_t* conv;        /* [n]                                             */
  uint8_t* stall;       /* [n]                                             */
  uint8_t* diverged;    /* [n]  post-hoc frozen-proposal probe             */
  float* stall_dchi2;   /* [n]  plateau certificate (NaN if not stalled)   */
  int32_t* nst;         /* [n]                                             */
  float* lam;           /* [n]                                             */
  int32_t* consec;      /* [n]                                             */
  int32_t* nrej;        /* [n]                                             */
  int64_t* n_good;      /* [n]  unmasked pixels summed over bands          */
  int32_t steps_run;    /* LM iterations executed for the chunk            */
  float* bg;            /* [n*nb*3] planar background (1, X, Y) per band
                           when bg_joint; may be NULL                      */
  float* bg_err;        /* [n*nb*3] its sqrt(diag inv A64); may be NULL    */
  int32_t* n_same;      /* [n]     "changed" tracker (0 otherwise); may be NULL */
  float* prej;          /* [n*N*6] last rejected proposal; may be NULL     */
  uint8_t* railed;      /* [n] trust region: a kept member parameter sits
                           at its box bound (island_solver.py:1717-1728);
                           0 in clip mode; may be NULL                     */
  float* perr;          /* [n*N*13] with param_errors: per member var of
                           (x, y, logre, ee1, ee2, u), cov(ee1, ee2), and
                           the six prior fractions pinv^2/(H_kk + pinv^2)
                           (NaN without priors); frozen and padded slots
                           read variance 1; NaN-filled without
                           param_errors; may be NULL                       */
  float* femarg;        /* [n*nb*N] with flux_marg: the increment (0 for
                           star rows and padded slots); NaN-filled
                           without flux_marg; may be NULL                  */
  float* smetrics;      /* [n*N*4] with source_metrics: rchisq, fracflux,
                           fracin, fracmasked (padded slots NaN, 0, NaN,
                           0); NaN-filled without; may be NULL             */
  float* swin;          /* [n*nb*N] with source_metrics: f * sum(m) per
                           band (NaN for padded slots); may be NULL        */
  float* reprof;        /* [n*N*12] with re_profile: chi2(p + dk e_logre)
                           - chi2(p); 0 for star and padded slots; NaN-
                           filled without; may be NULL                     */
  float* resid;         /* [n*B*B] with residual: sum_b w (d - model)      */
  float* resid_w;       /* [n*B*B] with residual: sum_b w; both NaN-filled
                           without; may be NULL                            */
  float* acond;         /* [n*nb] mixed precision: conditioning indicator
                           of each band's member normal matrix at the
                           final parameters (the spread of the f64
                           elimination's pivots of the diagonally scaled
                           matrix, the tensor-core routing test); NaN in
                           the plain form; may be NULL                     */
} uph_chunk_out;

/* Context: one per device per process. */
int uph_create(int device, uph_ctx** out);
int uph_destroy(uph_ctx* ctx);
const char* uph_last_error(const uph_ctx* ctx);
/* Optional: run on a caller-owned cudaStream_t (NULL = the context's own). */
int uph_set_stream(uph_ctx* ctx, void* stream);
void* uph_get_stream(const uph_ctx* ctx);

/* Padded field stacks (n_bands, Hp, Wp) float32: data - bg and inverse
 * variance (masked pixels 0); ``pad`` is the border width.  Copied to HBM.
 * A chunk added to a job binds the field, PSF and Sersic table the context
 * holds at that moment, and keeps them while the job lives: a later upload
 * of any of them to the context allocates fresh buffers instead of
 * overwriting ones a live chunk holds (and reuses them in place otherwise).
 * One job may therefore hold the chunks of several fields, each solved
 * against its own field and PSF -- requests packed into one solve. */
int uph_upload_field(uph_ctx* ctx, const float* data, const float* invvar,
                     int32_t n_bands, int32_t Hp, int32_t Wp, int32_t pad);
/* Same from device pointers (copied device-to-device). */
int uph_upload_field_device(uph_ctx* ctx, const float* data_dev,
                            const float* invvar_dev, int32_t n_bands,
                            int32_t Hp, int32_t Wp, int32_t pad);
/* Same stacks from the UNPADDED host field (nb, H, W): the padded
 * (nb, H + 2 pad, W + 2 pad) stacks are zeroed and filled on the device, so
 * the caller builds no padded host copy (the reference pads on the host,
 * island_solver.py:3334-3344). */
int uph_upload_field_unpadded(uph_ctx* ctx, const float* data, const float* invvar,
                              int32_t nb, int32_t H, int32_t W, int32_t pad);

/* Pixelised polynomial PSF zero-padded to tier T: coefs (n_bands, T, T, nt)
 * float32, origin_scale (n_bands, 4) = (x_origin, x_scale, y_origin,
 * y_scale).  One upload per tier. */
int uph_upload_psf_poly(uph_ctx* ctx, int32_t tier, const float* coefs,
                        const float* origin_scale, int32_t n_bands,
                        int32_t nt);

/* Analytic Gaussian-mixture PSF: params (n_bands, K, 4, nt) float32 holding
 * the polynomial coefficients of (sigma, e1, e2, weight) per component;
 * origin_scale as above. */
int uph_upload_psf_mog(uph_ctx* ctx, const float* params,
                       const float* origin_scale, int32_t n_bands, int32_t K,
                       int32_t nt);

/* Field-stack build: subtract each pass-1 tile's frozen planar background
 * from the context's uploaded data stack, on the device (the reference does
 * it on the host, island_stage.py:1728-1751).  tiles: n_tiles x (x0, y0,
 * x1, y1) core rectangles in unpadded pixels, applied in order; coefs:
 * (n_tiles, n_bands, M) float32 with M = 1, 3, 6 for order 0, 1, 2 and the
 * terms of make_bg_basis (bg_polynomial.py:125-178): 1, X, Y, X^2, XY,
 * Y^2 with X = (x - x_origin) / x_scale, Y = (y - y_origin) / y_scale in
 * float64, each term rounded to float32, summed by float32 fused
 * multiply-adds in term order; norm =
 * (x_origin, x_scale, y_origin, y_scale).  The field must not be held by a
 * live job (UPH_ERR_STATE): upload it, subtract, then add chunks. */
int uph_subtract_tile_backgrounds(uph_ctx* ctx, int32_t n_tiles, const int32_t* tiles,
                                  const float* coefs, int32_t order, const double* norm);

/* Field-wide scene subtraction of the star models (island_stage.py:
 * 2024-2118): for every band and every source i with flux[i, b] != 0,
 * flux[i, b] times its stamp -- the band's polynomial PSF (coefs (n_bands,
 * T, T, nt), origin_scale (n_bands, 4)) at the float32 position, Lanczos-3
 * shifted by the position's fractional part, not renormalised -- is
 * subtracted from the context's padded data stack at the corner
 * (round(x) - T/2, round(y) - T/2) + pad (round half to even of the
 * float64 position), clipped to the stack; product and difference each in
 * float32.  A pixel under several stamps is reduced in source order, as
 * the reference's loop (disjoint stamps run together).  The caller passes
 * the sources to subtract (the reference: the STAR members of the fit set;
 * extended sources stay in).  The field must not be held by a live job. */
int uph_scene_subtract_stars(uph_ctx* ctx, int32_t n, const double* x, const double* y,
                             const float* flux, int32_t T, int32_t nt, const float* coefs,
                             const float* origin_scale);
/* The wave of each source in that subtraction (host only, no device):
 * one more than the latest wave among the earlier sources whose T x T
 * stamps overlap its own; returns the number of waves, -1 on bad input. */
int uph_scene_waves(int32_t n, const double* x, const double* y, int32_t T, int32_t* wave);

/* Copy the context's padded field stacks (n_bands, Hp, Wp) float32 to host
 * buffers (either may be NULL). */
int uph_download_field(uph_ctx* ctx, float* data, float* invvar);

/* The "direct" backend's exponential mixture: k amplitudes and variances
 * (unit effective radius), float32. */
int uph_upload_exp_mog(uph_ctx* ctx, const float* amp, const float* var, int32_t k);

/* Sersic MoG table: knots [n_knots], amps/log_vars [n_knots*kmax], core
 * [n_knots], all float64. */
int uph_upload_sersic_table(uph_ctx* ctx, const double* knots,
                            const double* amps, const double* log_vars,
                            const double* core, int32_t n_knots,
                            int32_t kmax, double n_min, double n_max);

/* Fit one chunk of one class for up to max_steps LM iterations (host
 * buffers; the copies to and from the device are inside the call). */
int uph_run_chunk(uph_ctx* ctx, const uph_class_desc* cls,
                  const uph_chunk_in* in, int32_t max_steps,
                  uph_chunk_out* out);

/* Timing split of the last uph_run_chunk / uph_job_solve on the context
 * (milliseconds of device time between events): [0] host->device inputs,
 * [1] LM loop, [2] post-loop probes and final fluxes, [3] device->host
 * outputs. */
int uph_last_timing(const uph_ctx* ctx, float* ms4);

/* Number of kernel launches issued by the last uph_run_chunk / job solve. */
int64_t uph_last_launch_count(const uph_ctx* ctx);

/* ---- Jobs: many chunks (of any classes) resident on the device at once.
 * This is island_fit's class loop (island_solver.py:3380-3484) with every
 * chunk's inputs uploaded first and all chunks solved concurrently on a
 * pool of streams.  uph_job_solve may be called again: it restarts every
 * chunk from its uploaded inputs. */
typedef struct uph_job uph_job;
int uph_job_create(uph_ctx* ctx, uph_job** out);
int uph_job_destroy(uph_job* job);
/* Upload one chunk's inputs (host buffers); returns its index in *chunk_id. */
int uph_job_add_chunk(uph_job* job, const uph_class_desc* cls,
                      const uph_chunk_in* in, int32_t* chunk_id);
/* Solve every chunk for up to max_steps LM iterations (device-resident). */
int uph_job_solve(uph_job* job, int32_t max_steps);
/* LM loop engine of uph_job_solve.  UPH_ENGINE_QUEUE: every LM iteration
 * runs for all chunks of a lane at once, one kernel per kernel kind over a
 * device work queue of (chunk, island, unit) items; the queue holds the
 * islands still iterating, compacted on the device at the start of each
 * iteration from a longest-first order, and one CUDA graph per iteration is
 * launched per lane.  Its CTAs stay resident and pull units from an atomic
 * counter until the queue is empty.  UPH_ENGINE_QUEUE_PER_CTA: the same
 * queue with one unit per CTA (the grid covers the lane's units; CTAs past
 * the active ones exit at once).  UPH_ENGINE_CHUNKS (the default): each
 * chunk's iterations run as its own CUDA graph on one of a pool of streams.
 * All compute every island identically (bitwise the same results); the
 * queue engines need every chunk of the job to share the background mode
 * and otherwise fall back to the per-chunk engine.  Replaces the vmapped
 * chunk step of island_solver.py:1730-1752 with its width probe
 * (island_solver.py:2257). */
#define UPH_ENGINE_CHUNKS 0
#define UPH_ENGINE_QUEUE 1
#define UPH_ENGINE_QUEUE_PER_CTA 2
/* lanes (queue engine): the chunks are dealt to this many lanes, longest
 * processing time first, each with its own stream, work lists and iteration
 * graph, so that the lanes' phases overlap on the device (0: the default of
 * 8; at most 32). */
int uph_job_set_engine(uph_job* job, int32_t engine, int32_t lanes);
/* Copy one chunk's results to host buffers. */
int uph_job_read(uph_job* job, int32_t chunk_id, uph_chunk_out* out);
/* Per-kernel device time of the last instrumented solve: kind in
 * 0 render, 1 gram (FP32), 2 assemble, 3 step, 4 trial chi2, 5 accept,
 * 6 gram on the tensor cores; returns total milliseconds and launch count.
 * Instrumentation is on when uph_job_set_profile(job, 1) was called before
 * the solve.  An instrumented solve runs every chunk on one stream with
 * CUDA events around each launch (no graphs); its results are identical. */
#define UPH_KERNEL_KINDS 7
int uph_job_set_profile(uph_job* job, int32_t on);
int uph_job_kernel_time(const uph_job* job, int32_t kind, float* ms,
                        int64_t* launches);
/* Algorithmic work of the same kernels over the last instrumented solve, as
 * counted by every working CTA: bytes (stamps written by the render; stamp
 * rows over their member boxes, data, weights and the result for the Gram
 * and the trial chi2; small per-island arrays for the rest) and flops (the
 * Gram's K (K + 1) per window pixel; the step's 2/3 nL^3 LU; the render's
 * FP32 multiply-adds: per support pixel and Gaussian term reaching the tile
 * 4 + 4 x (derivative rows), per shifted array and pixel 14 for the Lanczos
 * passes, or the PSF polynomial in the pixelised-PSF mode). */
int uph_job_kernel_work(const uph_job* job, int32_t kind, double* bytes,
                        double* flops);
/* Exponential evaluations (SFU) of the same kernels over the last
 * instrumented solve: for the render, one per support pixel and Gaussian
 * term that reaches the pixel's tile (analytic mode). */
int uph_job_kernel_exps(const uph_job* job, int32_t kind, double* exps);

/* Compute-pipe peaks of the context's device for the roofline of the
 * kernels above (independent dependency chains over every SM, CUDA events,
 * best of three launches, about 10 ms in all): out[0] FP32 multiply-add
 * rate in TFLOP/s, out[1] exp2f evaluations in 10^12/s, out[2] FP64
 * multiply-add rate in TFLOP/s.  Allocates and frees a small device buffer.
 * No counterpart in the reference. */
int uph_measure_peaks(uph_ctx* ctx, double* out);
/* Device time from the start of the last uph_job_solve to the end of one
 * chunk's work (its LM iterations, probes and final pass), in ms. */
int uph_job_chunk_time(const uph_job* job, int32_t chunk_id, float* ms);

/* ---- Per-grid sparse forced photometry of one band ----------------------
 * Replaces solve_band_sparse (forced_phot_sparse.py:690-718, solver_inner
 * :498-555, assemble_and_solve :443-496) for point sources: every source's
 * PSF stamp at its fixed full-image position (psf_polynomial.py:134-197),
 * renormalised to unit sum when `renorm`, Lanczos-3 shifted by the
 * fractional grid-local position and placed at rint - half the stamp; the
 * weighted normal matrix of stamps and the polynomial background (order 0,
 * 1, 2: 1, 3, 6 terms X^m Y^n, X = (full-image x - x_origin) / x_scale),
 * stamp-overlap pairs taken from the caller's neighbour list
 * (build_neighbor_list, :272-330) and scatter-added; ridge
 * reg * max(|diag|, 1e-30) per diagonal element; a float64 solve and the
 * diagonal of the inverse.  Host arrays in and out. */
typedef struct uph_sparse_band {
  int32_t band_h, band_w;
  const float* data;          /* [band_h*band_w]                             */
  const float* invvar;        /* [band_h*band_w]                             */
  const uint8_t* pix_good;    /* [band_h*band_w] 0 = masked                  */
  int32_t n_sources;
  const float* pos_x;         /* [n] full-image pixel coordinates            */
  const float* pos_y;
  int32_t grid_x0, grid_y0;   /* this grid's top-left in the full image      */
  const float* psf_coefs;     /* [psf_h*psf_w*psf_nterms]                    */
  int32_t psf_h, psf_w, psf_nterms;
  float psf_x_origin, psf_x_scale, psf_y_origin, psf_y_scale;
  int32_t renorm;             /* 1: unit-sum stamps (the reference default)  */
  double bg_x_origin, bg_x_scale, bg_y_origin, bg_y_scale;
  int32_t bg_order;           /* 0, 1 or 2                                   */
  int32_t k_max;
  const int32_t* neighbor_idx;   /* [n*k_max], -1 where unused            */
  const uint8_t* neighbor_mask;  /* [n*k_max]                              */
  float reg;
  /* Extended sources ("fft" backend, source_model.py:304-318; may be NULL:
   * all stars): type (0 star, 1 EXP, 2 DEV, 3 SERSIC), ln Re, ee1, ee2 and
   * the Sersic index the mixture table is read at.  Galaxies need the
   * table (uph_upload_sersic_table); with any galaxy the stamps are not
   * renormalised, as the reference's mixed renderer. */
  const int32_t* source_type;
  const float* logre;
  const float* ee1;
  const float* ee2;
  const float* sersic_n;
  /* "direct" backend (source_model.py:218-256, 298-303) when render_direct
   * is 1: EXP sources are the exp_k-Gaussian mixture exp_amp / exp_var
   * sampled at pixel centres around the stamp centre, normalised, convolved
   * with the PSF stamp (same size, centred as mode "same") and renormalised
   * to unit sum; only STAR and EXP types are accepted and no Sersic table is
   * read.  0: the "fft" backend above. */
  int32_t render_direct;
  int32_t exp_k;              /* 1..16                                        */
  const float* exp_amp;       /* [exp_k]                                      */
  const float* exp_var;       /* [exp_k]                                      */
} uph_sparse_band;

typedef struct uph_sparse_out {
  float* fluxes;      /* [n]                                                  */
  float* bg_coefs;    /* [M]                                                  */
  float* flux_var;    /* [n] diagonal of the inverse normal matrix            */
  float* bg_var;      /* [M]                                                  */
  int32_t converged;  /* 1 when every flux and coefficient is finite          */
} uph_sparse_out;

int uph_sparse_band_solve(uph_ctx* ctx, const uph_sparse_band* in, uph_sparse_out* out);

/* ---- Island decomposition ------------------------------------------------
 * Replaces the coupled-pair search and connected-components labelling of
 * build_islands (islands.py:361-470, 423-560): sources i and j couple when
 * dist(i, j) < r_i + r_j (float64); rows flagged in forced_singleton (may
 * be NULL) couple with nothing.  root_out[i] = the minimum source index of
 * i's island, so islands ordered by root are the reference's deterministic
 * labels.  Positions and radii must be finite, radii positive. */
int uph_island_roots(uph_ctx* ctx, const double* pos_x, const double* pos_y,
                     const double* radius, const uint8_t* forced_singleton,
                     int32_t n, int32_t* root_out);

/* Attempts the union-find makes to link two coupled sources' roots before it
 * gives up (default UPH_ISLAND_TRIES_DEFAULT; each lost attempt means another
 * thread re-linked one of the roots first).  When a pair runs out the call
 * returns UPH_ERR_TIMEOUT and root_out is not a valid labelling; the context
 * stays usable.  0 makes any coupled pair that is not yet linked run out, so
 * the error path can be exercised on demand.  No counterpart in the
 * reference (its host cKDTree search has no retry loop). */
#define UPH_ISLAND_TRIES_DEFAULT (1 << 20)
int uph_set_island_retry_limit(uph_ctx* ctx, int32_t tries);

/* ---- Allocation-free final-flux pass.  No counterpart in the reference:
 * it exists for callers that cannot call cudaMalloc (a host inside a
 * framework that owns the device memory pool, or a serving process that
 * must not allocate after start-up).  Every buffer is a caller-owned DEVICE
 * pointer; the intermediates live in one fixed device array of
 * UPH_NOALLOC_SCRATCH_BYTES inside the library.  Star members, reference
 * render mode: renders each member at parameters p, solves the per-band
 * VarPro fluxes and returns fluxes, sqrt(diag inv A64) and the island chi2
 * -- the same numbers as uph_run_chunk with max_steps = 0.
 * Each island is checked on the device first: its real members must occupy
 * the leading member slots (at least one), all be SOURCE_STAR (0), and sit
 * within a stamp of the window; the window (bbox x bbox at ox, oy) must lie
 * inside the padded field.  An island that fails a check is not rendered
 * and its fluxes, ferr and chi2 come back NaN; the other islands are
 * unaffected.
 * Calls share the array: calls that overlap on the GPU race and must be
 * serialised by the caller.  The first call on a device does a one-time
 * set-up (the array's device address, kernel limits).  With CUDA's lazy
 * module loading (the default since CUDA 12.2) that first call is also when
 * the driver loads the library's kernels and commits the array's device
 * memory, so make it at start-up, before the memory budget is fixed and
 * before any stream capture.  Work that does not fit the array is rejected
 * with UPH_ERR_INVALID and a message in err_buf; later calls never allocate
 * and do not synchronise (results are ready when `stream` is). */
#define UPH_NOALLOC_SCRATCH_BYTES (32u << 20)
typedef struct uph_noalloc_args {
  const float* data;             /* (n_bands, Hp, Wp) padded field, data - bg */
  const float* invvar;           /* (n_bands, Hp, Wp)                       */
  const float* psf_coefs;        /* (n_bands, tier, tier, nt)               */
  const float* psf_origin_scale; /* (n_bands, 4)                            */
  const int32_t* ox;             /* [n] window origins in the padded field  */
  const int32_t* oy;             /* [n]                                     */
  const float* x0b;              /* [n] window origins in field coords      */
  const float* y0b;              /* [n]                                     */
  const int32_t* stype;          /* [n*N] SOURCE_STAR (0) for real members  */
  const uint8_t* mmask;          /* [n*N]                                   */
  const float* p;                /* [n*N*6] parameters (x, y used)          */
  float* fluxes;                 /* [n*n_bands*N] out                       */
  float* ferr;                   /* [n*n_bands*N] out                       */
  float* chi2;                   /* [n] out                                 */
  int32_t n_islands, nsrc, bbox, tier, native_stamp, n_bands, Hp, Wp, nt;
  float reg;                     /* ridge on real members (1e-9)            */
  void* stream;                  /* cudaStream_t (NULL = legacy default)    */
  char* err_buf;                 /* optional message buffer                 */
  int32_t err_len;
} uph_noalloc_args;
int uph_fluxes_noalloc(const uph_noalloc_args* args);

#ifdef __cplusplus
}
#endif
#endif /* UNIPHOT_B200_H */
