/*
 * bbmg_b200.h -- C ABI of the B200 black-box multigrid pressure solver.
 *
 * Drop-in for NGA2's bbmg pressure solve behind its linear-solver interface:
 *   init    -> bbmg_create   (ils_class.f90:162-226, bbmg_class.f90:185-600)
 *   setup   -> bbmg_setup    (ils_class.f90:230-256, 373-376; bbmg_class.f90:932-962)
 *   solve   -> bbmg_solve    (ils_class.f90:674-822;  bbmg_class.f90:604-728)
 *   destroy -> bbmg_destroy  (ils_class.f90:826-920)
 * The public linsol fields (linsol_class.f90:16-58) map to arguments: stc and
 * opr to bbmg_setup; rhs, sol, maxit, rcvg, it and rerr to bbmg_solve.
 *
 * Arrays use NGA2's Fortran layout: i fastest, then j, then k, each direction
 * padded by `ghost` overlap layers (the config's `no`).  The operator is
 * opr(nst, imino_:imaxo_, jmino_:jmaxo_, kmino_:kmaxo_) with the stencil index
 * fastest, exactly the caller's psolv%opr.  Only interior entries are read;
 * the solver copies in and out (ils_class.f90:247-256, 693-700, 782-788), so
 * caller arrays stay caller-owned.  Pointers may be host or device memory; the
 * kind is detected per call.
 *
 * Every entry point returns a status code and never aborts the host process.
 * A handle serves one stream and is not thread-safe; separate handles are
 * independent.  All compute runs on the GPU: there is no CPU fallback.
 */
#ifndef BBMG_B200_H
#define BBMG_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define BBMG_OK          0  /* converged: rerr <= rcvg                          */
#define BBMG_MAXIT       1  /* stopped at maxit without reaching rcvg          */
#define BBMG_STAGNATION  2  /* reserved: mixed precision falls back to FP64    */
#define BBMG_NONFINITE   3  /* NaN or Inf appeared in the residual             */
#define BBMG_BAD_ARGS    4  /* invalid argument (also a stencil outside 3x3x3) */
#define BBMG_NOT_SETUP   5  /* solve before setup (ils_class.f90:684)          */
#define BBMG_CUDA        6  /* a CUDA call failed; see bbmg_last_error         */
#define BBMG_NO_MEMORY   7  /* device allocation failed                        */

/* solution methods, NGA2's ILS ids (ils_class.f90:16-17) */
#define BBMG_METHOD_BBOX      1  /* stationary V-cycles (mgsolve)              */
#define BBMG_METHOD_PCG_BBOX  2  /* V-cycle preconditioned CG (cgsolve)        */

/* arithmetic of the solve */
#define BBMG_PREC_FP64   0  /* every step in FP64, the reference's arithmetic   */
#define BBMG_PREC_MIXED  1  /* FP32 V-cycle inside an FP64 outer iteration; when
                               the residual falls by < 10 % over 3 iterations the
                               solve continues with the FP64 method.  pcg_bbox
                               then updates its directions by the flexible rule
                               beta = -z.Ap_old / p_old.Ap_old (FCG(1)), since the
                               FP32 V-cycle is not an exactly symmetric fixed
                               preconditioner                                 */

typedef struct bbmg_handle bbmg_handle;

/* Grid: the pgrid sizes and periodicity bbmg reads (bbmg_class.f90:211-253). */
typedef struct {
    int nx, ny, nz;        /* interior cells per direction (>= 1)            */
    int xper, yper, zper;  /* periodicity flags                              */
    int ghost;             /* overlap layers of the caller's arrays (>= 0)   */
} bbmg_grid;

/* Solver knobs: the bbmg parameters the ILS sets (ils_class.f90:189-196,
 * bbmg_class.f90:91-98) plus the arithmetic mode. */
typedef struct {
    int method;            /* BBMG_METHOD_BBOX or BBMG_METHOD_PCG_BBOX       */
    int precision;         /* BBMG_PREC_FP64 or BBMG_PREC_MIXED              */
    int ncycle;            /* 1 = V-cycle, 2 = W-cycle                       */
    int relax_pre;         /* pre-smoothing sweeps                           */
    int relax_post;        /* post-smoothing sweeps                          */
    int ncell_coarsest;    /* coarsest level size limit                      */
    int use_direct_solve;  /* LU at the coarsest level (else relaxation)     */
    int maxit;             /* linsol maxit                                   */
    double rcvg;           /* linsol rcvg: relative inf-norm residual        */
    int device;            /* CUDA device ordinal; -1 = the current device   */
} bbmg_params;

/* Diagnostics of the last setup/solve. */
typedef struct {
    int nlvl;              /* levels in use                                  */
    int level_dims[16][3]; /* interior sizes per level (first nlvl rows)     */
    int coarse_n;          /* unknowns of the dense coarsest problem         */
    int coarse_pinned;     /* round-off pivots pinned in its LU (singular)   */
    int it;                /* iterations of the last solve                   */
    double rerr;           /* reported relative residual (inf-norm ratio)    */
    double res0;           /* initial residual inf-norm                      */
    double true_rerr;      /* max|b - A x| / (rerr's denominator), with x the
                              returned solution and the product recomputed in
                              FP64 after the last iteration (the reported rerr
                              of pcg_bbox is the CG recurrence's residual)   */
    double setup_ms;       /* device time of the last setup                  */
    double solve_ms;       /* device time of the last solve                  */
    long long device_bytes;/* device memory held by the handle               */
    int status;            /* status of the last solve                       */
    long long launches;    /* kernel launches of the last solve              */
    int level1_stencil;    /* level-1 storage: 27, 7, or 4 (symmetric 7-pt)  */
    int fallback_it;       /* mixed precision: iteration after which the solve
                              continued in FP64 because the FP32 V-cycle stopped
                              reducing the residual (0 = never)               */
    double true_res;       /* max|b - A x| at exit (absolute, FP64)           */
    double l2_rerr;        /* ||b - A x||_2 / ||r0||_2 at exit, r0 the initial
                              residual (||rhs||_2 under BBMG_NORM_RHS)        */
    int stage_it;          /* iterations that applied the preconditioner stage
                              (bbmg_set_precond_stage) in the last solve      */
} bbmg_info;

/* Fill `p` with the ILS values: pcg_bbox, FP64, V(2,2), ncell_coarsest 300,
 * direct coarsest solve, maxit 100, rcvg 1e-10, current device. */
void bbmg_default_params(bbmg_params *p);

/* init: build the level hierarchy and allocate device storage.
 * Replaces bbmg_from_pgrid + initialize (bbmg_class.f90:185-600) as called
 * from ils%init (ils_class.f90:184-198). */
int bbmg_create(const bbmg_grid *grid, const bbmg_params *params, bbmg_handle **handle);

/* setup: copy the caller's operator and rebuild every level.
 * stc is int[nst][3] (C order, the Fortran stc(st,1:3) transposed); every
 * offset must lie in [-1,1]^3.  opr is (nst, nx+2g, ny+2g, nz+2g), Fortran
 * order.  Replaces the ils scatter (ils_class.f90:244-256) and bbmg%update
 * (bbmg_class.f90:932-962). */
int bbmg_setup(bbmg_handle *h, int nst, const int *stc, const double *opr);

/* solve: rhs and sol are (nx+2g, ny+2g, nz+2g) Fortran arrays; sol holds the
 * initial guess on entry and the solution on exit (interior only; ghosts are
 * left for the caller's own sync).  it and rerr follow the reference's
 * definitions (bbmg_class.f90:627-633, 694-697, 721-724): rerr is
 * max|r|/max|r0| of the iteration's residual.  Either may be NULL.
 * Replaces ils%solve's bbmg branch (ils_class.f90:674-822). */
int bbmg_solve(bbmg_handle *h, const double *rhs, double *sol, int *it, double *rerr);

/* Change maxit / rcvg between solves (the linsol fields). */
int bbmg_set_convergence(bbmg_handle *h, int maxit, double rcvg);

/* Denominator of rerr.  BBMG_NORM_GUESS (default) is the reference's
 * max|r0| of the given initial guess (bbmg_class.f90:627-628), under which a
 * better guess cannot save iterations.  BBMG_NORM_RHS uses max|rhs|, the
 * residual a zero guess starts from: a solve from a predicted or warm-start
 * guess then stops at the same max|b - A x| as the zero-guess solve NGA2's
 * callers make (its zero-guess result is identical under both).  With a zero
 * rhs the solve falls back to max|r0|. */
#define BBMG_NORM_GUESS 0
#define BBMG_NORM_RHS   1
int bbmg_set_residual_norm(bbmg_handle *h, int norm);

/* First stage of a two-stage preconditioner for pcg_bbox in mixed precision.
 * The reference preconditions its CG with one V-cycle from a zero guess
 * (bbmg_class.f90:657-662); with a stage set, the preconditioner of an
 * iteration is z = S(r) + V(r - A S(r)): the caller's function S gives a first
 * approximation of A^-1 r (a learned network, for one), the FP32 V-cycle
 * corrects what it leaves, and the residual r - A S(r) is formed in FP64.  The
 * directions are A-orthogonalised against the previous one explicitly
 * (flexible CG, FCG(1)), so S may be nonlinear and change between calls.
 * r and z are the caller's device arrays of nx*ny*nz doubles (Fortran order,
 * no overlap layers) on the handle's device: before each call of fn the solver
 * writes the residual into r; fn(ctx, r, z, stream) writes z = S(r), enqueues
 * its work on `stream` (a cudaStream_t) and returns 0 (any other value ends
 * the solve with BBMG_BAD_ARGS); the solver reads z back.  `iters` = number of
 * leading iterations that apply the stage (0 = all); later iterations use the
 * V-cycle alone.  If the residual falls by less than 10 % over three
 * iterations, the solve continues as the plain FP64 pcg_bbox from the current
 * iterate (bbmg_info.fallback_it), so plain multigrid stays the fallback and
 * decides convergence.  fn = NULL removes the stage.  The handle must be
 * BBMG_METHOD_PCG_BBOX with BBMG_PREC_MIXED.  No counterpart in the
 * reference. */
typedef int (*bbmg_stage_fn)(void *ctx, const double *r, double *z, void *stream);
int bbmg_set_precond_stage(bbmg_handle *h, bbmg_stage_fn fn, void *ctx, int iters, double *r, double *z);

/* Run on the given cudaStream_t.  The default is a stream the handle
 * creates that synchronises with the legacy default stream, so device arrays
 * written there before a call are complete when the call reads them; with any
 * other producer stream, pass it here (or synchronise before the call). */
int bbmg_set_stream(bbmg_handle *h, void *stream);

int bbmg_get_info(const bbmg_handle *h, bbmg_info *info);

/* destroy: release the handle and its device memory. */
int bbmg_destroy(bbmg_handle *h);

/* Message of the last failure on this handle ("" if none); h may be NULL
 * for failures of bbmg_create. */
const char *bbmg_last_error(const bbmg_handle *h);

/* ------------------------------------------------------------------------
 * Step-level access, used by the parity tests to compare each stage of the
 * method with the reference's routine of the same name.  Arrays are exchanged
 * in the reference's own layout: one overlap layer, cell-major (k, j, i) with
 * the coefficient index fastest (27 for opr/f2c/oprc2f as opr(-1:1,-1:1,-1:1),
 * 8 for c2f as c2f(0:1,0:1,0:1)).
 * ---------------------------------------------------------------------- */
#define BBMG_ARR_OPR     0
#define BBMG_ARR_C2F     1
#define BBMG_ARR_F2C     2
#define BBMG_ARR_OPRC2F  3
#define BBMG_ARR_V       4
#define BBMG_ARR_F       5
#define BBMG_ARR_R       6

#define BBMG_STEP_RELAX        0  /* arg = +1/-1: relax(v, f, n, dir)      bbmg_class.f90:848-887 */
#define BBMG_STEP_RESIDUAL     1  /* get_residual(n)                       bbmg_class.f90:831-844 */
#define BBMG_STEP_RESTRICT     2  /* f2c(r_n -> f_n+1), v_n+1 = 0          bbmg_class.f90:805-827,739 */
#define BBMG_STEP_PROLONG      3  /* c2f(v_n+1 -> r_n); v_n += r_n         bbmg_class.f90:779-801,770 */
#define BBMG_STEP_CYCLE        4  /* cycle(n)                              bbmg_class.f90:732-776 */
#define BBMG_STEP_DIRECT       5  /* direct_solve()                        bbmg_class.f90:891-927 */

/* prec selects the FP64 (0) or FP32 (1) copy of a level's data.  The overlap
 * of f2c and oprc2f is read by nothing in the setup or the solve; on levels
 * with even sizes the setup leaves it unfilled, and bbmg_debug_get fills it
 * (zero in non-periodic directions, the periodic image otherwise, as the
 * reference holds it) on the handle's stream before the copy out. */
long long bbmg_debug_get(bbmg_handle *h, int level, int which, int prec, double *out);
long long bbmg_debug_put(bbmg_handle *h, int level, int which, int prec, const double *in);
int bbmg_debug_step(bbmg_handle *h, int step, int level, int arg, int prec);
/* Device time of one stage, for roofline measurements: the stage runs `reps`
 * times back to back on the handle's stream between two CUDA events; returns
 * the average milliseconds per repetition in *ms.  BBMG_STEP_RELAX times one
 * sweep as the V-cycle runs it (by colour phases on 7-point levels);
 * BBMG_STEP_CYCLE times cycle(level) as the solve runs it, the single-launch
 * coarse levels included. */
int bbmg_profile_step(bbmg_handle *h, int step, int level, int arg, int prec, int reps, double *ms);
/* dense coarsest matrix (row-major np x np), its LU (row-major, unit lower
 * below the diagonal) and pivots; any pointer may be NULL. */
int bbmg_debug_direct(bbmg_handle *h, double *op, double *lu, int *piv, int *np);

/* ------------------------------------------------------------------------
 * Residual check without device allocation.  No counterpart in the
 * reference: it serves callers that cannot call cudaMalloc -- a flow solver
 * whose device memory comes from its own pool allocator, or a time loop that
 * must not allocate because allocation can synchronise the device.
 *
 * Computes, on `stream` (NULL: the default stream), out[0] = max|rhs - A sol|,
 * out[1] = max|rhs| and out[2] = out[0] / out[1] over the interior of the
 * caller's system, with A the caller's stencil (stc host array int[nst][3],
 * opr in bbmg_setup's layout), overlap cells of non-periodic directions taken
 * as zero and periodic directions wrapped.  out[2] is the rerr bbmg_solve
 * reports for a solve that started from a zero guess (its max|r0| is then
 * max|rhs|); for a zero rhs out[2] is 0 if the residual is 0, else +inf.
 * opr, rhs, sol and out (3 doubles) must be memory of the current device.
 * Nothing is allocated: the only scratch is a static device array of 8192
 * plane slots that every GPU loading the library holds until exit, so grids
 * with nz > 8192 are rejected with BBMG_BAD_ARGS.  Each call looks up that
 * array's address on the current device; under CUDA's lazy module loading the
 * first call on a device also loads the library's device code there, which can
 * synchronise the device, so make one warm-up call before a time loop or any
 * stream capture.  Calls share the array: calls that overlap on the GPU race
 * and must be serialised by the caller.  Errors: bbmg_last_error(NULL).
 * ---------------------------------------------------------------------- */
int bbmg_residual_norm_noalloc(const bbmg_grid *grid, int nst, const int *stc, const double *opr,
                               const double *rhs, const double *sol, double *out, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* BBMG_B200_H */
