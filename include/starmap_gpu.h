/*
 * starmap_gpu.h -- C ABI of the B200 (sm_100a, FP64) time-stepping library
 * that replaces the time loop of StaRMAP's starmap_solver(par).
 *
 * The reference is MATLAB/GNU Octave.  Its solver function
 *     output = starmap_solver(par)            (starmap_solver.m:1)
 * keeps its host-side setup (starmap_solver.m:55-157: flags, grid-type
 * classification, staggered grids, hook sampling, first-step materials,
 * decay factors, source and filter tables, starmap_solver.m:165-305) and hands
 * the arrays to this library once; the library runs the whole Strang-split loop
 * (starmap_solver.m:307-421) on one GPU and returns the final components.
 * A MEX/oct gateway, a ctypes binding or any other FFI binds these symbols:
 * only plain pointers, sizes and POD structs cross the boundary.
 *
 * Conventions
 *   - Every entry point returns SMG_OK (0) or a negative SMG_E* code; the
 *     message of the last failure on a handle is smg_last_error(handle), and
 *     of a failed smg_create / handle-less call smg_last_error(NULL).  The
 *     handle-less message is kept per host thread: the pointer stays valid
 *     until the same thread's next handle-less failure.  No C++ exception
 *     leaves the library: host memory exhausted inside a call returns
 *     SMG_ENOMEM, any other C++ exception SMG_EINVAL, with its message.
 *   - Arrays follow MATLAB's column-major order.  Component j lives on the
 *     staggered grid gt[3*j+d] (1 = cell centres, 2 = staggered points) and
 *     has extent n[d] along solver dimension d, or n[d]+1 when gt == 2 and
 *     bc[d] == 1 (starmap_solver.m:113-126).
 *   - Components and fields are 0-based here (component 0 = MATLAB U{1}).
 *   - Host buffers are borrowed for the duration of the call only.
 *   - A handle is used by one host thread at a time.  All GPU work of a
 *     handle runs on its own CUDA stream; entry points that return host data
 *     synchronise that stream.
 */
#ifndef STARMAP_GPU_H
#define STARMAP_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* The library is built with hidden default visibility; everything declared
 * here is exported. */
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#define SMG_OK          0
#define SMG_EINVAL     -1   /* inconsistent or unsupported input (MATLAB would error()) */
#define SMG_ECUDA      -2   /* CUDA runtime/launch failure */
#define SMG_ETIMEOUT   -3   /* a bounded device wait gave up (batched grid barrier) */
#define SMG_ENONFINITE -4   /* non-finite state detected by smg_check_finite */
#define SMG_ENOMEM     -5   /* device or host allocation failed */
#define SMG_ESTATE     -6   /* call out of order (e.g. run before the state is set) */

#define SMG_VARIANT_AUTO    0  /* best available kernel family (JIT, else pair, else strip); phase A fused (default) */
#define SMG_VARIANT_GENERIC 1  /* point-per-thread kernels, one launch per half step */
#define SMG_VARIANT_STRIP   2  /* strip kernels, one launch per half step */
#define SMG_VARIANT_STAGED  3  /* strip kernels, slot-job loads staged by cp.async; phase A fused */
#define SMG_VARIANT_PAIR    4  /* two points per thread, destination-centric; phase A fused */
#define SMG_VARIANT_JIT     5  /* pair layout, kernels generated for this problem and compiled at run time (NVRTC) */

#define SMG_FILTER_NONE    0   /* par.f_position = ''          */
#define SMG_FILTER_SUBSTEP 1   /* par.f_position = 'substep'   */
#define SMG_FILTER_FULL    2   /* par.f_position = 'full'      */

typedef struct smg_handle smg_handle;

/* One coefficient array of the solver: sT1{g,m}, ET{g,m}, sA1, EA, Q{j} or a
 * filterTerm{g,m[,k]}.  data == NULL means the reference held a scalar
 * (hooks may return scalars, which MATLAB broadcasts); otherwise data points to
 * a column-major array with the extents of grid `grid`. */
typedef struct smg_field {
    const double* data;
    double scalar;
    int32_t grid[3];            /* grid type per solver dimension, 1 or 2 */
} smg_field;

/* Problem descriptor: everything starmap_solver.m holds when it enters the
 * update loop at starmap_solver.m:307. */
typedef struct smg_problem {
    int32_t n_sys;              /* number of moment components, length(par.Mz) */
    int32_t n[3];               /* par.n (solver ordering; 2D: [1 nx ny]) */
    int32_t bc[3];              /* par.bc: 0 periodic, 1 extrapolation */
    double  h[3];               /* grid spacing, starmap_solver.m:101 */
    const int32_t* gt;          /* [3*n_sys] grid type per component and dimension */
    const double* Mx;           /* [n_sys*n_sys] column-major par.Mx */
    const double* My;           /* [n_sys*n_sys] column-major par.My */
    const double* Mz;           /* [n_sys*n_sys] column-major par.Mz */
    int32_t n_fields;           /* number of entries in `fields` */
    const smg_field* fields;
    const int32_t* sigma_t;     /* [n_sys] field of sT1{gt(j),mom_order(j)} (entry 0 unused) */
    const int32_t* decay_t;     /* [n_sys] field of ET{...}, or NULL: computed on the GPU by smg_set_dt */
    int32_t sigma_a;            /* field of sA1 = sA{1,1,1} */
    int32_t decay_a;            /* field of EA, or -1: computed on the GPU by smg_set_dt */
    const int32_t* source;      /* [n_sys] field of Q{j}, -1 = zero (not in par.source_ind) */
    int32_t filter_mode;        /* SMG_FILTER_* */
    const int32_t* filter1;     /* [n_sys] filterTerm{..,k=1} (substep) or filterTerm (full); -1 = 1 */
    const int32_t* filter2;     /* [n_sys] filterTerm{..,k=2} (substep only); -1 = 1 */
} smg_problem;

/* Library version string. */
const char* smg_version(void);

/* Message of the last failure on `h` (or of the last handle-less failure). */
const char* smg_last_error(const smg_handle* h);

/* Number of visible CUDA devices (>= 0), or a negative SMG_E* code. */
int smg_device_count(void);

/* Select the CUDA device used by handles created afterwards on the calling
 * thread (one process per GPU: rank r calls smg_set_device(local_rank)). */
int smg_set_device(int32_t device);

/* Validate the descriptor, build the coupling tables (the Ix/Iy/Iz lists of
 * starmap_solver.m:77-79 in sumcell order, starmap_solver.m:350-351/398-399),
 * allocate device memory and upload the coefficient fields. Limits: n[d] <=
 * 2^30, and one component's padded slot (the points of the first kernel axis
 * rounded up to 8, times those of the other two, faces included) below 2^31
 * points, since the kernels index a point with 32 bits; else SMG_EINVAL.
 * Every coupling M_d(j,i) != 0 must join grid types that differ in axis d
 * alone (as smg_classify assigns them); else SMG_EINVAL.
 * Replaces: starmap_solver.m:136-157 (field allocation) on the device side. */
int smg_create(const smg_problem* p, smg_handle** out);

/* Release all device memory and the stream of `h`. */
void smg_destroy(smg_handle* h);

/* Upload the state: U[j] is the column-major host array of component j
 * (U{j} of starmap_solver.m:140-146).  Pointers may not be NULL.  Any host
 * memory works; page-locked arrays move fastest (see SMG_TUNE_DIRECT_XFER),
 * and an array page-locked only in part is copied through a host bounce
 * buffer.  The same holds for smg_get_state and smg_get_interp. */
int smg_set_state(smg_handle* h, const double* const* U);

/* Download the state into per-component host arrays; a NULL entry skips that
 * component (used for par.mom_output subsets).  Synchronises the stream. */
int smg_get_state(smg_handle* h, double* const* U);

/* Replace the values of one coefficient field (time-dependent sources,
 * materials or filters re-evaluated by the host between steps,
 * starmap_solver.m:214-252, 278-305). */
int smg_set_field(smg_handle* h, int32_t field, const double* data, double scalar);

/* Set the time step.  Decay factors not supplied by the host (decay_t NULL,
 * decay_a -1) are computed on the GPU as expm1div(-sigma*dt/2)
 * (starmap_solver.m:267-274, 531-535) at this point. */
int smg_set_dt(smg_handle* h, double dt);

/* Time of the current state (default 0): the start of the next smg_run when
 * sources are evaluated on the device (smg_set_source_expr); each step then
 * advances it by dt, as the reference's loop does (t = t + dt). */
int smg_set_time(smg_handle* h, double t);

/* Time-dependent source of component `comp` evaluated on the device: before
 * every step of smg_run the library writes Q_comp = expr at each point of the
 * component's grid, at the step's t - dt/2 (starmap_solver.m:276-282), then
 * runs the step; such runs are not fused across steps and use no CUDA graph.
 * `expr` is an arithmetic expression in C++ syntax (compiled with NVRTC for
 * sm_100a at the next smg_run; see smg_check_expr for what it may contain)
 * in x, y, z, t and k: the point's coordinates
 * in the three solver dimensions, the time and the 1-based component number
 * -- the arguments of the reference's source hook after starmap_init.
 * x/y/z hold the coordinates of the component's grid along each solver
 * dimension (its extent there, 1 for a singleton dimension).  The source must
 * be an array field of its own; expr = NULL returns to the uploaded values.
 * The reference evaluates a Matlab function on the host instead; this is the
 * device-evaluable form of that hook. */
int smg_set_source_expr(smg_handle* h, int32_t comp, const char* expr, const double* x, const double* y,
                        const double* z);

/* Kinds of device expressions, for smg_check_expr. */
#define SMG_EXPR_SOURCE   0   /* variables x, y, z, t, k */
#define SMG_EXPR_MATERIAL 1   /* variables x, y, z, t, m */
#define SMG_EXPR_FILTER   2   /* variables x, y, z, t, dt, k */

/* SMG_OK when `expr` is a valid device expression of `kind`, else SMG_EINVAL
 * with the reason in smg_last_error(NULL).  Device expressions are spliced
 * into generated kernels, so they are held to a grammar that cannot reach
 * memory or leave the expression: decimal or hexadecimal numbers, the kind's
 * variables, the math functions sin cos tan asin acos atan atan2 sinh cosh
 * tanh asinh acosh atanh exp exp2 exp10 expm1 log log2 log10 log1p pow sqrt
 * rsqrt cbrt hypot fabs abs fmin fmax min max fmod remainder floor ceil round
 * rint trunc copysign erf erfc tgamma lgamma sinpi cospi fdim nearbyint,
 * true, false, the operators + - * / % < > <= >= == != && || ! ?: and
 * parentheses and commas.  smg_set_source_expr, smg_set_material_expr and
 * smg_set_filter_expr refuse anything else with SMG_EINVAL. */
int smg_check_expr(int32_t kind, const char* expr);

/* Time-dependent materials evaluated on the device: before every step of
 * smg_run the library evaluates sigma_a, sigma_s0 and (expr_sm non-NULL)
 * sigma_sm at t + dt, forms sigma_t = sigma_a + (sigma_s0 - sigma_sm) per
 * (grid type, order), averages each with its values at t into the field and
 * writes its decay factor expm1div(-s dt/2) (starmap_solver.m:214-252,
 * 267-274); the values at t are taken at the first smg_run after
 * smg_set_time.  Expressions as for smg_set_source_expr, in x, y, z, t and,
 * for sigma_sm, the order m.  rows: nrows triples (sigma_t field, its decay
 * field, order m); sA_field / EA_field: sigma_a on grid 111 and its decay
 * field; all array fields.  coords: 6 vectors, per solver dimension the
 * coordinates of grid type 1 then 2.  expr_a = NULL returns to uploaded
 * values.  The reference evaluates Matlab hooks on the host instead. */
int smg_set_material_expr(smg_handle* h, const char* expr_a, const char* expr_s0, const char* expr_sm, int32_t nrows,
                          const int32_t* rows, int32_t sA_field, int32_t EA_field, const double* const* coords);

/* Time-dependent filter evaluated on the device: before every step of
 * smg_run the library writes, per row, the filter at t - dt/2 into field
 * rows[3r] and at t into rows[3r+1] ('substep'; rows[3r+1] = -1 for 'full':
 * at t into rows[3r]), for the row's order k = rows[3r+2]
 * (starmap_solver.m:283-305).  expr in x, y, z, t, dt and k, as for
 * smg_set_source_expr; coords as for smg_set_material_expr.  expr = NULL
 * returns to uploaded values.  The reference evaluates a Matlab hook on the
 * host instead. */
int smg_set_filter_expr(smg_handle* h, const char* expr, int32_t nrows, const int32_t* rows,
                        const double* const* coords);

/* Keep a copy of the current state on the device for smg_get_interp (the
 * first call allocates it; it is freed with the handle).  The reference keeps
 * that copy on the host (U0 before the last step of an output interval,
 * starmap_solver.m:425-430). */
int smg_snapshot(smg_handle* h);

/* The components j with U[j] non-NULL of (1 - lambda) * snapshot +
 * lambda * state, computed on the device in the reference's operation order
 * and written to host arrays as smg_get_state does: the linear interpolation
 * to an output time inside the last step (starmap_solver.m:431-473). */
int smg_get_interp(smg_handle* h, double lambda, double* const* U);

/* Advance `nsteps` full Strang steps A(dt/2) B(dt) A(dt/2) [+ full filter]
 * (starmap_solver.m:307-421) with the current dt.  Asynchronous on the
 * handle's stream; steps that move under 1 GB are replayed from captured
 * 64-step CUDA graphs, heavier ones are launched directly (SMG_TUNE_GRAPH_STEPS). */
int smg_run(smg_handle* h, int64_t nsteps);

/* Wait for all work of `h`. */
int smg_sync(smg_handle* h);

/* Choose the kernel family (SMG_VARIANT_*).  All variants produce identical
 * results; AUTO falls back to GENERIC when a schedule does not fit in shared
 * memory.  No reference counterpart (the reference has one CPU code path). */
int smg_set_variant(smg_handle* h, int32_t variant);

/* The kernel family the next smg_run uses (AUTO resolved; JIT only after it
 * was compiled: by smg_set_variant(JIT) or by AUTO's first smg_run) and, in
 * `why` (cap bytes, may be NULL), the form of the generated kernels when JIT
 * is active ("bulk-staged", "async-staged" or "register", SMG_TUNE_JIT_STAGED), else the
 * reason AUTO could not use JIT. */
int smg_active_variant(smg_handle* h, int32_t* variant, char* why, int64_t cap);

/* The CUDA C++ source of the specialised kernels (SMG_VARIANT_JIT) of problem
 * p, generated with the SMG_TUNE_JIT_* settings keys[i] = values[i] (ntune of
 * them; defaults otherwise); *len receives its length, buf (cap bytes) a
 * NUL-terminated copy.  compile = 1 also compiles it with NVRTC for sm_100a
 * (no GPU needed); compile = 2 adds (to the source and the compilation) the
 * adjoint's recording and backward-phase kernels, compile = 3 the batched
 * solver's family kernels.  SMG_EINVAL for a problem whose state holds 2^31
 * doubles or more (the generated kernels use 32-bit element offsets).  No
 * reference counterpart. */
int smg_jit_source(const smg_problem* p, const int32_t* keys, const int32_t* values, int32_t ntune, int32_t compile,
                   char* buf, int64_t cap, int64_t* len);

/* Process-wide counts of generated-kernel programs compiled with NVRTC and
 * of programs loaded from the on-disk cache instead.  Compiled kernels are
 * kept in $SMG_JIT_CACHE_DIR (else $XDG_CACHE_HOME/starmap_b200, else
 * $HOME/.cache/starmap_b200), keyed by their source, compile options and the
 * NVRTC and library versions, so that a new process (a new MATLAB session)
 * does not compile the same problem's kernels again; SMG_JIT_CACHE=0 turns
 * the cache off.  No reference counterpart. */
int smg_jit_stats(int64_t* compiled, int64_t* from_disk);

/* Tuning parameters of the kernels (no reference counterpart).  They change
 * performance only, never results.  Keys: */
#define SMG_TUNE_PAIR_GROUP  1   /* destinations per CTA of the pair kernel (1..256) */
#define SMG_TUNE_PAIR_BLOCK  2   /* threads per CTA of the pair kernel (32..256, multiple of 32) */
#define SMG_TUNE_PAIR_UNROLL 3   /* couplings per inner iteration (1 or 2) */
#define SMG_TUNE_PAIR_MINB   4   /* register budget: 3 or 4 resident CTAs of 256 threads (64/85 regs) */
#define SMG_TUNE_ADJ_FUSED   5   /* smg_backward: 1 = one fused kernel per phase (default), 0 = pointwise + transpose kernels */
#define SMG_TUNE_JIT_LANES   22  /* generated kernels of one phase that run at the same time: 0 (default) all of
                                    them, n >= 1 at most n (kernel i follows kernel i - n on its stream) */
#define SMG_TUNE_DIRECT_XFER 21  /* state transfers: 1 (default) separate page-locked host arrays are read / written
                                    in place by one kernel per 64 components, while arrays carved in order from one
                                    page-locked block (at most one contiguous run per eight arrays) and pageable
                                    ones go through the double-buffered device staging buffer, host-adjacent pieces
                                    in one copy; 0 always through the staging buffer */
#define SMG_TUNE_ADJ_PRIORITY 20 /* smg_backward stream priorities, set before smg_forward: 0 (default) recompute and
                                    sweep at the default priority, 1 recompute at the device's highest priority, 2
                                    the sweep on a stream of the highest priority above the recompute */
#define SMG_TUNE_JIT_BLOCK   6   /* threads per CTA of the generated kernels (32..256, multiple of 32; default: of
                                    64 and 96 the one leaving the fewest idle points in a row, 96 on ties) */
#define SMG_TUNE_JIT_GROUP   7   /* destinations per CTA of the generated kernels (1..256) */
#define SMG_TUNE_JIT_REGS    8   /* register limit per thread of the generated kernels (0: compiler's choice, else 32..255) */
#define SMG_TUNE_JIT_SPLIT   9   /* groups per separately compiled program (1..64; 0: one per phase) */
#define SMG_TUNE_JIT_CALLS  10   /* 0: one kernel per program, the kernels of a phase run concurrently (default);
                                    1: one kernel per phase calling the separately compiled groups */
#define SMG_TUNE_JIT_XPAIR  11   /* x differences: 0 = four 64-bit loads per point pair, 1 = two aligned 128-bit loads,
                                    2 = one 128-bit load and the neighbouring lane's value (warp shuffle) */
#define SMG_TUNE_JIT_PREFETCH 12 /* 1: the generated kernels request a group's rows into L2 before loading them;
                                    2, 3: each CTA's first thread requests into L2, with bulk prefetches, the row
                                    segments that the group 1 or 2 places later in the same kernel reads there */
#define SMG_TUNE_JIT_BAND   13   /* CTA order of the generated kernels: 0 group-major, R > 0 bands of R rows,
                                    -1 (default) group-major below 4 MB per component, else bands of about 48 MB;
                                    staged kernels: 0 group-major, else band-major (bands of SMG_TUNE_JIT_ROWS) */
#define SMG_TUNE_JIT_CONST  14   /* 1 (default): coupling weights and grid constants read from a __constant__ table; 0: immediates */
#define SMG_TUNE_GRAPH_STEPS 15  /* steps per captured CUDA graph of smg_run: 0 direct launches, no graph; -1 (default)
                                    direct launches when a step moves 1 GB or more, else 64 */
#define SMG_TUNE_JIT_STAGED 16   /* form of the generated kernels: 0 (default) loads to registers at first use; 1 each
                                    row's segments staged in a shared-memory ring by bulk copies (cp.async.bulk) from a
                                    producer thread; 2 the same ring filled by the consumer warps' 16-byte asynchronous
                                    copies; 3 the default form with a per-thread ring of asynchronous copies one
                                    destination ahead.  All give identical results; 1-3 measured slower. */
#define SMG_TUNE_JIT_SLICES 17   /* staged kernels: consumer warps per CTA, each taking a slice of a group (1..16) */
#define SMG_TUNE_JIT_STAGES 18   /* staged kernels: shared-memory ring depth in rows (2..6) */
#define SMG_TUNE_JIT_ROWS   19   /* staged kernels: rows per CTA (0: about eight waves of CTAs per phase) */
int smg_tune(smg_handle* h, int32_t key, int32_t value);

/* Kernel-only timing of the last smg_run (milliseconds, CUDA events on the
 * handle's stream) and its launch count. */
int smg_last_run_stats(smg_handle* h, double* ms, int64_t* launches);

/* Device bytes held by `h`, and the padded device layout of one component
 * (elements per row, rows per plane, planes, component stride). */
int smg_layout(const smg_handle* h, int64_t* bytes, int64_t dims_out[4]);

/* Scan the state for NaN/Inf on the GPU; returns SMG_ENONFINITE if any. */
int smg_check_finite(smg_handle* h);

/* Sum of squares of every component of the state, sumsq[n_sys] (host):
 * the squared discrete L2 norms monitored by starmap_2d_ex_l2norm.m:93-99
 * (which applies staggered trapezoid weights on top).  Deterministic order. */
int smg_state_sumsq(smg_handle* h, double* sumsq);

/* Sums of squares of ncomp device vectors without allocating any GPU memory.
 * No counterpart in the reference: it serves hosts that must not allocate on
 * the device themselves (a MEX gateway that only holds MATLAB-owned gpuArray
 * buffers, a caller under a fixed device-memory budget).  Vector c holds len
 * doubles at d_x + c*stride; d_out (device) receives ncomp sums; stream is a
 * cudaStream_t (NULL: the default stream).  The partial sums live in a fixed
 * 256 KB array inside the library, resident on every GPU that loads it, so
 * ncomp is limited to 1024 (larger requests return SMG_EINVAL).  The first
 * call on a device looks up that array's device address, and so does the
 * first call after the device's context was reset (cudaDeviceReset, MATLAB's
 * reset(gpuDevice)), since the array may then live elsewhere: make those
 * calls before any stream capture on that device.  All calls share the array: calls whose
 * GPU work overlaps (different streams or threads) race on it.  The message
 * of a failed call is smg_last_error(NULL). */
int smg_sumsq_noalloc(const double* d_x, int32_t ncomp, int64_t stride, int64_t len, double* d_out,
                      void* stream);

/* Spectral radius *la = max |eig(G_o G_e G_e G_o)| of the full-step growth
 * matrix that the parabolic time step searches over (starmap_solver.m:
 * 506-514, growth_factor): G is the n x n complex matrix
 * diag(dt*expm1div(-decay*dt/2)) * (M + diag(-decay/2)), column-major with
 * interleaved real and imaginary parts; odd[i] = 1 for the components that
 * phase A updates (their rows of G_e are identity rows, the other rows of
 * G_o are), 0 for phase B's.  The products run on the current device with
 * cuBLAS and the eigenvalues with cuSOLVER (cusolverDnXgeev), both opened
 * at the first call; synchronous.  Replaces the host eig of growth_factor;
 * errors through smg_last_error(NULL). */
int smg_growth_radius(int32_t n, const double* G, const int32_t* odd, double* la);

/* Grid-type classification of starmap_solver.m:76-98 from the sparsity of
 * par.Mx/My/Mz (column-major n_sys x n_sys): writes gt_out[3*j+d] in {1,2}.
 * SMG_EINVAL when a component is not reached from component 1 (the
 * reference's loop never ends there) or when a coupling along axis d joins
 * components whose grid types differ in more than axis d (the reference would
 * put a component on two grids).  Host-only helper for callers that do not
 * classify themselves. */
int smg_classify(int32_t n_sys, const double* Mx, const double* My, const double* Mz,
                 int32_t* gt_out);

/* ---------------------------------------------------------------------------
 * Discrete adjoint.  No reference counterpart (the reference has no
 * derivatives); it differentiates exactly the loop smg_run performs.
 * smg_forward(h, nsteps, K) advances nsteps steps from the current state and
 * keeps a checkpoint every K steps (K = 0: the largest K whose recording fits
 * in 70% of the free device memory, normally K = nsteps, which records the
 * whole run during the forward and recomputes nothing); the last segment is
 * recorded during the forward itself.  smg_misfit(h, obs, &J) evaluates
 * J = 1/2 sum (U_1(T) - obs)^2 on the zeroth moment (obs: host, component-0
 * extents) and seeds the adjoint with U_1(T) - obs (smg_adjoint_seed seeds
 * any adjoint state instead); smg_backward recomputes each segment from its
 * checkpoint and runs the transposed phases back to t = 0, returning
 * dJ/dU(0) per component and dJ/d(field) for every sigma and source field:
 * an array of the field's extents, or one number for a scalar field (the sum
 * over the points it acts on).  Decay fields are treated as
 * expm1div(-sigma*dt/2) of their sigma field (their derivative enters the
 * sigma gradient); filter fields are constants.  Requires f_position '' or
 * 'substep' and fields that stay fixed between smg_forward and smg_backward.
 * smg_last_run_stats after smg_forward / smg_backward reports the device
 * time of that call's GPU work (host copies of the results excluded).
 * --------------------------------------------------------------------------- */
int smg_forward(smg_handle* h, int64_t nsteps, int64_t ckpt_every);
int smg_misfit(smg_handle* h, const double* obs, double* J);
int smg_adjoint_seed(smg_handle* h, const double* const* lam);
/* grad_U0[j]: host array (component extents) or NULL; grad_fields[f]: host
 * array (array field) / one double (scalar field) / NULL, f < n_fields. */
int smg_backward(smg_handle* h, double* const* grad_U0, double* const* grad_fields);
/* Device bytes held for checkpoints and adjoint buffers. */
int smg_adjoint_bytes(const smg_handle* h, int64_t* bytes);
/* Segment length K and segment count of the last smg_forward (0, 0 before one). */
int smg_adjoint_info(const smg_handle* h, int64_t* K, int64_t* nseg);

/* ---------------------------------------------------------------------------
 * Batched solver: many problems (uneven grid sizes and moment orders, each
 * with its own dt) advanced together by one persistent cooperative launch per
 * block of steps, the launch sequence replayed from a CUDA graph.  No
 * reference counterpart: the reference solves one problem per call; a batch
 * replaces a host loop of starmap_solver calls.  Each instance is an ordinary
 * handle (state I/O through smg_batch_instance + smg_set_state/smg_get_state).
 * --------------------------------------------------------------------------- */
typedef struct smg_batch smg_batch;

#define SMG_BATCH_BLOCK            1  /* threads per CTA (32..256, multiple of 32) */
#define SMG_BATCH_GROUP            2  /* destinations per work item (1..256) */
#define SMG_BATCH_STEPS_PER_LAUNCH 3  /* Strang steps per persistent launch */
#define SMG_BATCH_SPIN_LIMIT       4  /* polls before a grid-barrier wait gives up (SMG_ETIMEOUT) */
#define SMG_BATCH_BARRIER_EXTRA    5  /* test hook: barrier expects one CTA more than launched (0/1) */
#define SMG_BATCH_USE_GRAPH        6  /* 1: replay the launch sequence from a CUDA graph */
#define SMG_BATCH_PERSISTENT       7  /* 1: one cooperative launch per block of steps; 0: one launch per phase */
#define SMG_BATCH_JIT              8  /* 1: kernels generated per family of equal-structure instances (default;
                                         built on the first run, NVRTC needed), 0: the precompiled kernels */

/* Instances with f_position 'full' (SMG_FILTER_FULL) are refused (SMG_EINVAL):
 * the batch kernels do not apply the full-step filter. */
int smg_batch_create(int32_t n_inst, const smg_problem* const* probs, smg_batch** out);
void smg_batch_destroy(smg_batch* b);
const char* smg_batch_last_error(const smg_batch* b);
/* Handle of instance i (owned by the batch; do not destroy). */
smg_handle* smg_batch_instance(smg_batch* b, int32_t i);
/* dt[i] for every instance (decay factors recomputed as by smg_set_dt). */
int smg_batch_set_dt(smg_batch* b, const double* dt);
/* Advance every instance by nsteps Strang steps; SMG_ETIMEOUT if a grid
 * barrier wait ran out of its spin limit (the state is then undefined). */
int smg_batch_run(smg_batch* b, int64_t nsteps);
int smg_batch_last_run_stats(smg_batch* b, double* ms, int64_t* launches);
int smg_batch_tune(smg_batch* b, int32_t key, int64_t value);
/* Current block, group, steps per launch and persistent grid size (0 when
 * the batch runs one launch per phase). */
/* Whether the last runs used the generated family kernels, and how many
 * families (sets of instances sharing kernels) the batch has. */
int smg_batch_info(const smg_batch* b, int64_t* jit_active, int64_t* families);
int smg_batch_config(const smg_batch* b, int64_t out[4]);
/* Time probe_steps steps for each candidate configuration (block x group x
 * steps per launch), keep the fastest; every instance's state is restored. */
int smg_batch_autotune(smg_batch* b, int64_t probe_steps, double* best_ms);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif

#endif /* STARMAP_GPU_H */
