/* fast_gpu.h - C ABI of libfastgpu.so, the B200 (sm_100a) implementation of
 * FAST's solid element-integration, assembly and K.u solve path.
 *
 * The library sits under FAST's own C++ interfaces.  Each entry point below
 * names the reference interface it replaces (file:line inside the FAST
 * tree).  Above it sits a C++ shim in FAST's own terms: a cSysMatrix
 * subclass whose virtuals forward here, and a batched
 * cControl::StiffnessMatrix that uploads the mesh once and assembles on the
 * device.
 *
 * Conventions
 *   - Every call returns an int status: FAST_GPU_OK (0) or a negative
 *     FAST_GPU_E* code; fast_gpu_last_error() gives a message.  No C++
 *     exception crosses this boundary.
 *   - Vectors passed as host pointers have length num_eq and follow FAST's
 *     equation numbering (cControl::CompEqs, ctrl/ctrl.cpp:2056-2104):
 *     entry k belongs to equation k+1.  They are what cVector::Val() gives.
 *   - Matrix indices (i, j) are 0-based equation indices, as in
 *     cSysMatrix::Add/Get (mlib/sysmat.h:85-86).
 *   - The context owns all device memory; one context serves one host thread.
 *   - Calls are stream-ordered on the context's stream; calls that return
 *     host data synchronise that stream.  Every device wait is bounded.
 */
#ifndef FAST_GPU_H
#define FAST_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FAST_GPU_ABI_VERSION 1

/* ---- status codes ---------------------------------------------------- */
#define FAST_GPU_OK         0
#define FAST_GPU_EINVAL    -1   /* bad argument                                  */
#define FAST_GPU_ENOMEM    -2   /* device or host allocation failed              */
#define FAST_GPU_ECUDA     -3   /* CUDA runtime error                            */
#define FAST_GPU_ESTATE    -4   /* call out of order (e.g. solve before assemble) */
#define FAST_GPU_ENONCONV  -5   /* solver reached maxit without convergence       */
#define FAST_GPU_EDETJ     -6   /* non-positive Jacobian determinant in an element */
#define FAST_GPU_ENOTSUP   -7   /* element type / option not supported           */
#define FAST_GPU_ENOTFOUND -8   /* (i, j) outside the sparsity pattern           */
#define FAST_GPU_ETOOBIG   -9   /* system larger than an entry point's fixed limit */

/* ---- element types (FAST readers elc/element.cpp:1985-2101) ----------- */
#define FAST_ELEM_HEX8      1   /* %ELEMENT.BRICK8   cElmParam,  SHAPE_BRICK8  */
#define FAST_ELEM_HEX20     2   /* %ELEMENT.BRICK20  cElmParam,  SHAPE_BRICK20 */
#define FAST_ELEM_BSP_SOLID 3   /* %ELEMENT.BSPLINE.SOLID cElmParam, SHAPE_BSP_SOLID: Bezier-extracted
                                   B-spline / NURBS solid (shp/shpbsp.cpp:873-1067); degrees
                                   (2,2,2) with 3 or 4 Gauss points per direction, (3,3,3) and
                                   (3,3,2) with 4, (4,2,4) and (4,2,2) with 5, (5,2,5) with 6;
                                   FAST_FORM_TOTAL_LAGRANGIAN (%ELEMENT.BSPLINE.SOLIDTL) for
                                   (2,2,2), (3,3,3), (3,3,2) and (4,2,2); the consistent mass
                                   (a density per element) for (2,2,2), (3,3,3), (3,3,2);
                                   needs a patch */

/* ---- element formulation --------------------------------------------- */
#define FAST_FORM_SMALL_STRAIN       0  /* cElmParam   (%ELEMENT.BRICK8 / BRICK20)     */
#define FAST_FORM_TOTAL_LAGRANGIAN   1  /* cElmParamTL (%ELEMENT.BRICK8TL / BRICK20TL),
                                           St. Venant-Kirchhoff, elc/elmparam.cpp:1615-1807 */

/* ---- what to assemble ------------------------------------------------- */
#define FAST_ASM_STIFFNESS  1   /* cControl::StiffnessMatrix (ctrl/ctrl.cpp:886-975); total-
                                   Lagrangian buckets give their tangent at the current
                                   displacements */
#define FAST_ASM_MASS       2   /* cControl::MassMatrix      (ctrl/ctrl.cpp:979-1027) */
#define FAST_ASM_INTERNAL_FORCE 3  /* element internal forces (fast_gpu_element_matrices only) */
#define FAST_ASM_STIFFNESS_TF32 4  /* the stiffness for the mixed-precision solve: element
                                      products B^T C B on the tensor cores (tcgen05, TF32 operands split in three,
                                      FP32 accumulation), blocks stored in FP32.  Small-strain
                                      hex8 / hex20 buckets and B-spline solids of degree (2,2,2),
                                      (3,3,3) or (3,3,2); elements touching a tied node keep FP64
                                      element matrices, scattered into the FP32 blocks.  The FP64 stiffness slot is
                                      then stale: fast_gpu_solve takes FAST_PREC_MIXED only and forms
                                      its FP64 residuals r = f - K u element by element in FP64
                                      (the small-strain internal force at u); the next
                                      FAST_ASM_STIFFNESS assembly restores the FP64 path. */

/* ---- solver precision ------------------------------------------------- */
#define FAST_PREC_FP64      0   /* FP64 Jacobi PCG, as PCGSolver (mlib/sysmat.cpp:1061-1125) */
#define FAST_PREC_MIXED     1   /* FP32 PCG, FP64 solution and residual replacement
                                   ("reliable updates"); continues in FP64 if the FP32
                                   iterates stall on an ill-conditioned system       */

/* ---- preconditioner --------------------------------------------------- */
#define FAST_PRECOND_JACOBI        0  /* z = r / diag(K), as the reference      */
#define FAST_PRECOND_BLOCK_JACOBI  1  /* z = inv(3x3 nodal block) r               */

typedef struct fast_gpu_ctx fast_gpu_ctx;

/* The B-spline patch of a FAST_ELEM_BSP_SOLID bucket (cBspPat, geom/patch.cpp:
 * 1459-1484, read from %PATCH; element spans from %ELEMENT.BSPLINE.SOLID,
 * shp/shpbsp.cpp:57-116).  The element's local nodes are its (p+1)^3 control
 * points with the r index fastest, then s, then t (cShapeBspSolid::Init,
 * shp/shpbsp.cpp:873-902). */
typedef struct {
  int32_t        degree[3];     /* polynomial degree per direction                      */
  int32_t        num_knots[3];  /* knot vector lengths, repeated knots included          */
  const double  *knots[3];      /* knot vectors with multiplicities expanded (cKnotVector::Val) */
  const int32_t *span;          /* [num_elems][3] 0-based non-zero knot span per direction */
  const double  *weights;       /* [num_nodes] control-point weights (%CONTROL.POINT.WEIGHT)
                                   or NULL for unit weights (cNode::GetW, node/node.cpp:656-662) */
  int32_t        rational;      /* patch rational flag: 1 = NURBS quotient N_a w_a / W,
                                   0 = plain tensor-product B-spline                        */
  int32_t        reserved;
} fast_gpu_patch;

/* One bucket = one element type with one Gauss rule (a FAST element reader
 * block with one %INTEGRATION.ORDER).  Material: isotropic linear elastic per
 * element (E, nu: cMatElastIso), the constitutive matrix of cSolid::QMatrix;
 * the element kernels fold it into the Gauss-point contraction, so a general
 * 6x6 tangent (cConstModel::TangMat of other material models) has no device
 * path. */
typedef struct {
  int32_t        elem_type;     /* FAST_ELEM_*                                 */
  int32_t        ngp[3];        /* Gauss points per direction (r, s, t)        */
  int64_t        num_elems;
  const int32_t *conn;          /* [num_elems][nn] 0-based node indices, FAST local order */
  const double  *E;             /* [num_elems] Young's modulus                 */
  const double  *nu;            /* [num_elems] Poisson's ratio                 */
  const double  *rho;           /* [num_elems] density, or NULL                */
  int32_t        formulation;   /* FAST_FORM_*                                 */
  int32_t        reserved;
  const fast_gpu_patch *patch;  /* FAST_ELEM_BSP_SOLID: its patch; NULL otherwise  */
} fast_gpu_bucket;

/* Tied interfaces between non-matching meshes.  Each tie is the three linear
 * constraints  u_s,i - sum_k w_k u_(m_k),i = 0  (i = x, y, z) of one slave node
 * s on the surface of its master elements; in the reference they are
 * %NODE.MULTI-POINT.CONSTRAINT equations (cNode::ReadNodeMPC, node/node.cpp:
 * 459-509) solved with dense Lagrange multipliers by cSysMatrix::SolveMPC
 * (mlib/sysmat.cpp:72-143).  Here the slave DOFs are eliminated: with u = T u~,
 * the library assembles K~ = T^T K T directly into the node-block matrix and
 * solves K~ u~ = T^T f; slave displacements are interpolated back.  A slave
 * must not be a master, and its equations (if any) stay in the caller's
 * numbering: loads on them are carried to the masters.  fast_gpu_get_lower_csr
 * and fast_gpu_mult_vect then see K~, with an identity diagonal on the slave
 * equations. */
typedef struct {
  int64_t        num_slaves;
  const int64_t *slave;         /* [num_slaves] tied nodes (0-based, distinct)        */
  const int64_t *ptr;           /* [num_slaves + 1] offsets into master / weight      */
  const int64_t *master;        /* master nodes of each slave                         */
  const double  *weight;        /* interpolation weights w_k                         */
} fast_gpu_ties;

typedef struct {
  int64_t                num_nodes;
  const double          *coords;    /* [num_nodes][3]                          */
  const int32_t         *node_eq;   /* [num_nodes][3] 1-based equation, 0 = fixed/unused */
  int32_t                num_eq;
  int32_t                num_buckets;
  const fast_gpu_bucket *buckets;
  const fast_gpu_ties   *ties;      /* NULL: no tied interfaces (linear statics only) */
} fast_gpu_mesh;

typedef struct {
  int32_t precision;      /* FAST_PREC_*                                        */
  int32_t precond;        /* FAST_PRECOND_*                                     */
  int32_t maxit;          /* iteration cap (total inner iterations); 0 = 20*num_eq */
  int32_t warm_start;     /* 1: start from the u passed in (mixed path: as the first iterate) */
  double  tol;            /* stop when |r|/|f| < tol (|f| > 1e11 replaced by 1, as the reference) */
  double  inner_tol;      /* reserved, 0                                          */
  int32_t max_outer;      /* reserved, 0                                          */
  int32_t check_every;    /* iterations per chunk: convergence read-back period and,
                             mixed, FP64 residual replacement period; 0 = 32 (FP64) / 50 (mixed) */
} fast_gpu_solve_opts;

typedef struct {
  int32_t converged;
  int32_t iterations;      /* PCG iterations (FP32 + FP64 iterations when mixed)  */
  int32_t outer;           /* FP64 residual replacements (mixed), 1 for FP64        */
  int32_t escalated;       /* mixed: bit 0 FP32 iterates stalled, finished in FP64; bit 1 the tensor-core
                              stiffness stalled, the FP64 stiffness was assembled and the mixed
                              iteration went on with it */
  double  rel_residual;    /* |r|/|f| of the final FP64 residual (mixed) or recurrence (FP64) */
  double  true_rel_residual; /* |f - K u| / |f| recomputed in FP64 at exit           */
} fast_gpu_solve_report;

/* ---- lifetime ---------------------------------------------------------- */
int         fast_gpu_create(int device, fast_gpu_ctx **ctx);
int         fast_gpu_destroy(fast_gpu_ctx *ctx);
const char *fast_gpu_last_error(const fast_gpu_ctx *ctx);
int         fast_gpu_version(void);
/* Use a caller's CUDA stream (a cudaStream_t passed as void*); NULL = context's own. */
int         fast_gpu_set_stream(fast_gpu_ctx *ctx, void *cuda_stream);
int         fast_gpu_synchronize(fast_gpu_ctx *ctx);
/* Tuning options (no reference counterpart). */
#define FAST_OPT_PERSISTENT_MAX_NODES 1  /* PCG on systems with at most this many nodes runs each chunk
                                            of iterations as one persistent cooperative kernel (grid
                                            barriers instead of kernel boundaries); default 65536,
                                            0 = always one kernel per step of the iteration */
#define FAST_OPT_SPMV_LANES_FP32      2  /* lanes per block-row of the FP32 SpMV: 4, 8 (default), 16, 32 */
#define FAST_OPT_SPMV_LANES_FP64      3  /* lanes per block-row of the FP64 SpMV: 4, 8, 16 (default), 32 */
#define FAST_OPT_SPMV_BULK_FP32       5  /* 1: the FP32 SpMV streams the matrix through shared memory by
                                            bulk copies (tiles of block-rows, two stages); 0 (default
                                            until fast_gpu_autotune measures it): register loads */
#define FAST_OPT_GRAPH_STEPS          4  /* 1 (default): fast_gpu_newmark replays every step after the first
                                            as one CUDA graph, and fast_gpu_nr_solve every Newton
                                            iteration after a step's first (the PCG loop inside as a
                                            conditional WHILE node); 0: launch kernel by kernel */
#define FAST_OPT_ZERO_FILL            7  /* 0 (default): where every block of the pattern is reached by an
                                            element (no tied interfaces, no total-Lagrangian buckets), the
                                            stiffness assembly stores each block at its first write instead
                                            of zero-filling K and adding to it; 1: zero-fill all the same */
#define FAST_OPT_SPMV_STREAM_FP32     9  /* 1: the FP32 SpMV loads the matrix with cache-streaming (evict-
                                            first) loads, 8 or 16 lanes per row; 0 (default until
                                            fast_gpu_autotune measures it): plain loads */
#define FAST_OPT_SPMV_COL16_FP32     10  /* 1: the FP32 SpMV reads 16-bit column offsets from each row's
                                            smallest column (38 instead of 40 bytes per block; every row
                                            must span fewer than 65,536 nodes, else FAST_GPU_ENOTSUP);
                                            0 (default until fast_gpu_autotune measures it): 32-bit */
#define FAST_OPT_FORCE_GATHER        11  /* 1 (default): where every bucket is a hex bucket, the internal
                                            force is formed element by element in one launch per bucket
                                            and gathered per node in the order the colour-by-colour
                                            scatter adds it (the same bits); 0: one launch per colour */
#define FAST_OPT_PERSISTENT_ASSEMBLY  8  /* 1: FAST_ASM_STIFFNESS_TF32 integrates the elements of every
                                            bucket in one persistent cooperative launch (colour k of
                                            every bucket is phase k, grid barriers between phases, CTAs
                                            take elements from a counter, heaviest kinds first); 0
                                            (default): one launch per bucket and colour */
#define FAST_OPT_ELEM_SHAPE           6  /* launch shape of one bucket's element kernels, value =
                                            kernel << 32 | bucket << 24 | tc_ctas << 16 | split << 8 | ctas
                                            (each field 0..255, 0 = the default): resident CTAs per SM of
                                            the FP64 kernels (ctas) and of the tensor-core kernels
                                            (tc_ctas), CTAs sharing one B-spline element (split), the FP64
                                            hex stiffness kernel (0 one CTA per element, 1 one warp per
                                            element); what fast_gpu_autotune chooses, for callers that
                                            cache its choices */
int         fast_gpu_set_option(fast_gpu_ctx *ctx, int32_t option, int64_t value);

/* Autotuner (no reference counterpart): times, per bucket of small-strain
 * elements, the stiffness assembly for every launch shape of its element
 * kernels (resident CTAs per SM; for B-spline buckets also the CTAs that
 * share one element) on the FP64 path and, where every bucket has one, on the
 * tensor-core path (CUDA events, median of 3 assemblies each), then
 * re-assembles K with the chosen shapes; times the SpMV of the assembled
 * stiffness for every lanes-per-row choice in both precisions (median of 9
 * launches each), chooses the FP32 SpMV form by 64 mixed PCG iterations with
 * each (median of 3) and, for systems small enough for the persistent PCG kernel,
 * one 64-iteration FP64 PCG chunk on each iteration path; keeps the fastest
 * choices as the context's options.  Needs an assembled K; uses the solver's
 * work vectors (call it before a solve, not during one). */
typedef struct {
  int32_t lanes_fp32, lanes_fp64;       /* chosen lanes per block-row                      */
  double  ms_fp32[4], ms_fp64[4];       /* per launch for 4, 8, 16, 32 lanes              */
  int64_t persistent_max_nodes;         /* chosen limit for the persistent PCG kernel     */
  double  us_iter_persistent, us_iter_kernels;  /* FP64 PCG per iteration, or 0 if not timed */
  double  ms_fp32_bulk[2];              /* bulk-staged FP32 SpMV per launch, 8 and 16 lanes per row */
  int32_t bulk_fp32;                    /* 1: the bulk-staged FP32 SpMV was kept                  */
  int32_t reserved;
  int32_t elem_buckets;                 /* buckets reported below (the first 8; TL buckets untimed)  */
  int32_t elem_tc;                      /* 1: the tensor-core kernels were timed too                 */
  int32_t elem_ctas[8], elem_split[8], elem_tc_ctas[8];  /* chosen shapes (0 = default)             */
  double  elem_ms_default[8], elem_ms_tuned[8];          /* FP64 stiffness of the bucket, per assembly */
  double  elem_tc_ms_default[8], elem_tc_ms_tuned[8];    /* tensor-core stiffness of the bucket      */
  double  ms_fp32_stream[2];            /* FP32 SpMV with cache-streaming matrix loads, 8 and 16 lanes   */
  int32_t stream_fp32;                  /* 1: the cache-streaming FP32 SpMV was kept                      */
  int32_t reserved2;
  double  us_iter_mixed[6];             /* mixed PCG per iteration with each FP32 form (the choice):
                                           8 / 16 lanes plain, cache-streaming, bulk-staged (0: not run) */
  double  us_iter_mixed_col16[2];       /* the same with 16-bit column offsets, 8 / 16 lanes (0: not run) */
  int32_t col16_fp32;                   /* 1: the 16-bit column offsets were kept                        */
  int32_t reserved3;
  int32_t elem_kernel[8];               /* FP64 hex stiffness kernel chosen per bucket: 0 one CTA per
                                           element, 1 one warp per element                            */
} fast_gpu_tune_report;
int         fast_gpu_autotune(fast_gpu_ctx *ctx, fast_gpu_tune_report *rep);

/* ---- mesh and pattern ---------------------------------------------------
 * Replaces cControl::Init's CompEqs/CompProf (ctrl/ctrl.cpp:2004-2157) for the
 * device matrix: copies the mesh, builds the node-block (3x3) CSR pattern,
 * the element-to-block slot map and a greedy element colouring. */
int fast_gpu_upload_mesh(fast_gpu_ctx *ctx, const fast_gpu_mesh *mesh);
int fast_gpu_pattern_info(fast_gpu_ctx *ctx, int64_t *nnz_blocks, int64_t *nnz_lower_eq,
                          int32_t *num_colors, double *pattern_seconds);
/* Same topology, new values (host buffers of the upload's sizes). */
int fast_gpu_update_coords(fast_gpu_ctx *ctx, const double *coords);
int fast_gpu_update_material(fast_gpu_ctx *ctx, int32_t bucket, const double *E, const double *nu);

/* ---- displacement state and internal force ----------------------------
 * cControl::AssignDispl (ctrl/ctrl.cpp:1094-1113): the nodal displacements
 * the total-Lagrangian tangent and the internal force are evaluated at
 * (equation space, length num_eq; initially zero). */
int fast_gpu_set_displacement(fast_gpu_ctx *ctx, const double *u);
int fast_gpu_set_displacement_device(fast_gpu_ctx *ctx, const double *d_u);
/* cControl::IntForceVector (ctrl/ctrl.cpp:719-813): g = sum of element
 * internal forces at the current displacements (cElmParam::IntForce
 * elc/elmparam.cpp:449-535, cElmParamTL::IntForce :1615-1707). */
int fast_gpu_internal_force(fast_gpu_ctx *ctx, double *g);
int fast_gpu_internal_force_device(fast_gpu_ctx *ctx, double *d_g);

/* ---- load-control Newton-Raphson ----------------------------------------
 * cCtrlNR::Solver (ctrl/ctrlnr.cpp:47-270) with proportional loading on the
 * device: per step f = lambda q; per iteration tangent at u, K du = r,
 * u += du, g = IntForce(u), r = f - g, converged when |r|/max(1,|f|) < tol
 * (cControl::Convergence, ctrl/ctrl.cpp:1366-1413).  Each step starts from
 * the last converged u (FAST_NR_PREDICT_NONE, the reference), from the secant
 * extrapolation 2u_k - u_{k-1}, or from a caller's prediction, taken only when
 * its residual is smaller than the secant start's. */
#define FAST_NR_PREDICT_NONE      0
#define FAST_NR_PREDICT_SECANT    1
#define FAST_NR_PREDICT_CALLBACK  2

typedef struct {
  int32_t steps;              /* MAXIMUM.STEPS                                       */
  int32_t max_iter;           /* MAXIMUM.ITERATIONS                                  */
  double  step_factor;        /* STEP.FACTOR (load increment)                        */
  double  tol;                /* TOLERANCE                                           */
  int32_t predictor;          /* FAST_NR_PREDICT_*                                   */
  int32_t reserved;
  fast_gpu_solve_opts lin;    /* linear solves K du = r                             */
  double  lin_tol_rel;        /* > 0: inexact Newton, linear tol = clamp(max(lin_tol_rel *
                                 err, tol / (2 err)), lin_tol_min, lin_tol_max) with err
                                 the current Newton error; 0: lin.tol as given        */
  double  lin_tol_min, lin_tol_max;
} fast_gpu_nr_opts;

typedef struct {
  int32_t converged_steps;
  int32_t failed_step;        /* 0, or the step that did not converge                */
  int32_t iterations;         /* Newton iterations (tangent assemblies), all steps    */
  int32_t linear_iterations;  /* PCG iterations, all steps                           */
  int32_t secant_starts, predictions, predictions_accepted, reserved;
  double  last_err;           /* |r|/max(1,|f|) at the last iteration                */
  double  last_rel_residual;  /* |r|/|f| at the last iteration                       */
} fast_gpu_nr_report;

/* Caller predictor: write the predicted u at load factor lambda (step >= 2)
 * into d_u_pred (device, equation space) and return 0, or return non-zero to
 * skip.  d_u_last / d_u_prev are the last two converged solutions, d_f the
 * external load of this step (lambda q).  The context's displacement state
 * may be changed by the predictor. */
typedef int (*fast_gpu_nr_predictor)(void *user, int32_t step, double lambda, const double *d_u_last,
                                     const double *d_u_prev, const double *d_f, double *d_u_pred);

/* q: reference load (host, num_eq).  u_hist (host, [steps][num_eq]) and iters
 * ([steps], -1 for a failed step) may be NULL. */
int fast_gpu_nr_solve(fast_gpu_ctx *ctx, const double *q, const fast_gpu_nr_opts *opts,
                      fast_gpu_nr_predictor predictor, void *predictor_user, double *u_hist, int32_t *iters,
                      fast_gpu_nr_report *rep);

/* ---- modal analysis ------------------------------------------------------
 * cCtrlModal::Solver (ctrl/ctrlmodal.cpp:48-128) with the subspace iteration
 * of cGenEigSubSpaces::Solver (mlib/eig.cpp:377-510): M and K assembled on
 * the device, q = max(2p, p + 8) vectors (at most 32, so p <= 16), each
 * iteration K Y = M X by PCG, the projected pencil Y^T K Y, Y^T M Y solved on
 * the host, X = Y Phi; converged when sqrt(|1 - lambda^2 / |phi|^2|) <= tol for
 * the p lowest, the reference's measure.  lambda [num_modes] are the
 * eigenvalues (natural frequencies sqrt(lambda)); modes [num_modes][num_eq]
 * (may be NULL) the M-normalised mode shapes, sign arbitrary.  Needs
 * densities in every bucket (fast_gpu_bucket.rho). */
typedef struct {
  int32_t num_modes;          /* EIGEN.NUMBER.MODES (the reference's default is 5)  */
  int32_t max_iter;           /* MAXIMUM.ITERATIONS of the subspace loop             */
  double  tol;                /* TOLERANCE on the reference's convergence measure    */
  fast_gpu_solve_opts lin;    /* the K solves (tol relative to the right-hand side)  */
} fast_gpu_modal_opts;

typedef struct {
  int32_t converged;
  int32_t iterations;         /* subspace iterations                                 */
  int32_t linear_iterations;  /* PCG iterations, all solves                          */
  int32_t subspace;           /* q                                                   */
  double  max_err;            /* the convergence measure at the last iteration        */
} fast_gpu_modal_report;

int fast_gpu_modal(fast_gpu_ctx *ctx, const fast_gpu_modal_opts *opts, double *lambda, double *modes,
                   fast_gpu_modal_report *rep);

/* Linear buckling: cCtrlLinStab::Solver (ctrl/ctrllinstab.cpp:46-140).
 * K u = f (f host, num_eq: the reference load), the geometric stiffness G
 * at u assembled on the device (cControl::GeomStiffMatrix ctrl/ctrl.cpp:
 * 1031-1063, cElmParam::GeomStiff elc/elmparam.cpp:743-830), then the same
 * subspace iteration on K v = lambda (-G) v.  lambda ascending as the
 * reference orders them (a state with tension can give negative factors
 * first); modes normalised v^T (-G) v = 1; u (num_eq, may be NULL) gets the
 * linear solution.  opts.lin serves the linear solve and the iteration's
 * solves.  Small-strain hex buckets; the mass slot is overwritten (the next
 * mass assembly rebuilds it). */
int fast_gpu_buckling(fast_gpu_ctx *ctx, const double *f, const fast_gpu_modal_opts *opts, double *lambda,
                      double *modes, double *u, fast_gpu_modal_report *rep);

/* ---- path following (arc length) ---------------------------------------
 * cCtrlPath::Solver (ctrl/ctrlpath.cpp:63-265) with the load-increment rules
 * of the reference's arc-length classes (ctrl/ctrlarclen.cpp:95-250), on the
 * device: per iteration the tangent at u, K du1 = q and K du2 = r (two PCG
 * solves on unit right-hand sides), the rule's load increment dlf,
 * du = dlf du1 - du2, r = g(u) - lambda q, converged when
 * |r| / max(1, |q|) < tol (cControl::Convergence, ctrl/ctrl.cpp:1366-1380).
 * The arc length is StepFactor (|du1| + LoadCoeff) at the first step and is
 * scaled by sqrt(TargetIter / iterations of the last step) afterwards
 * (%HEADER.ANALYSIS.ARC-LENGTH gives LoadCoeff, TARGET.ITERATIONS TargetIter,
 * whose reference default is 1).  No strain loads, critical points or large
 * rotations (the reference's options around this loop). */
#define FAST_ARC_INITIAL_NORMAL 1   /* 'ioal'   cIniOrtArcLength */
#define FAST_ARC_UPDATED_NORMAL 2   /* 'uoal'   cUpOrtArcLength  */
#define FAST_ARC_LINEARIZED     3   /* 'clinal' cConLinArcLength */

typedef struct {
  int32_t method;             /* FAST_ARC_*                                          */
  int32_t steps;              /* MAXIMUM.STEPS                                       */
  int32_t max_iter;           /* MAXIMUM.ITERATIONS                                  */
  int32_t target_iter;        /* TARGET.ITERATIONS (0: keep the arc length)          */
  double  step_factor;        /* STEP.FACTOR: first load increment                   */
  double  tol;                /* TOLERANCE                                           */
  double  load_coeff;         /* ARC-LENGTH load coefficient                          */
  fast_gpu_solve_opts lin;    /* the inner solves (tol relative to the unit rhs)     */
} fast_gpu_arc_opts;

typedef struct {
  int32_t converged_steps;
  int32_t failed_step;        /* 0, or the step that did not converge                */
  int32_t iterations;         /* tangent assemblies, all steps                       */
  int32_t linear_iterations;  /* PCG iterations, all steps                           */
  double  last_err;           /* |r| / max(1, |q|) at the last iteration              */
  double  arc_length;         /* at the last step                                    */
} fast_gpu_arc_report;

/* q: reference load (host, num_eq).  u_hist (host, [steps][num_eq]),
 * lambda_hist ([steps]) and iters ([steps]) may be NULL. */
int fast_gpu_arclength_solve(fast_gpu_ctx *ctx, const double *q, const fast_gpu_arc_opts *opts, double *u_hist,
                             double *lambda_hist, int32_t *iters, fast_gpu_arc_report *rep);

/* ---- learned load-step predictor ------------------------------------------
 * No counterpart in the reference (cCtrlNR starts every step from the last
 * converged u).  A POD basis Phi (num_eq x modes) of converged displacements
 * and a tanh MLP that maps the load factor lambda_s and the last `history`
 * coefficient sets (a = Phi^T u), given as a_{s-1} and its history-1 backward
 * differences, each scaled per mode, to the in-basis correction of the secant
 * increment:
 *   u_pred = u_{s-1} + rho (u_{s-1} - u_{s-2}) + Phi (tau * mlp(x)),
 * rho = dlambda_s / dlambda_{s-1}.  The network trains and runs on the
 * device with BF16 tensor-core GEMMs accumulating in FP32; the POD is FP64.
 * fast_gpu_ws_predict has the fast_gpu_nr_predictor signature: pass it with
 * the predictor object as user to fast_gpu_nr_solve (FAST_NR_PREDICT_CALLBACK);
 * fast_gpu_nr_solve takes the prediction only when its residual is below the
 * secant start's, and Newton iterates to the same tolerance either way. */
typedef struct fast_gpu_ws fast_gpu_ws;

typedef struct {
  int32_t modes;        /* POD modes k (e.g. 32)                                 */
  int32_t history;      /* coefficient sets in the network input (e.g. 4)       */
  int32_t width;        /* hidden layer width (e.g. 256)                         */
  int32_t hidden;       /* hidden layers (e.g. 2: in -> 256 -> 256 -> k)         */
  int32_t oversample;   /* range-finder columns beyond k (e.g. 16)               */
  int32_t power_iters;  /* range-finder power iterations (e.g. 2)                */
  uint64_t seed;        /* initial weights and range-finder test matrix          */
} fast_gpu_ws_opts;

typedef struct {
  int32_t trajectories, snapshots, samples, modes;
  int32_t input_dim, output_dim, epochs, reserved;
  int64_t params;
  double captured_energy;   /* sum of the kept squared singular values / |S|_F^2 */
  double basis_ms, train_ms;
  float  first_loss, last_loss;
  int64_t launches;         /* kernels launched by the predictor object           */
  int64_t predictions, galerkin_iterations;
  double predict_ms;        /* host time inside fast_gpu_ws_predict               */
} fast_gpu_ws_stats;

/* The predictor lives on ctx's device and stream; ctx must hold a mesh. */
int fast_gpu_ws_create(fast_gpu_ctx *ctx, const fast_gpu_ws_opts *opts, fast_gpu_ws **out);
void fast_gpu_ws_destroy(fast_gpu_ws *ws);
/* One training trajectory: the converged u of every load step (host,
 * [steps][num_eq], e.g. fast_gpu_nr_solve's u_hist) and its load factors. */
int fast_gpu_ws_add_trajectory(fast_gpu_ws *ws, int32_t steps, const double *lambda, const double *u_steps);
/* POD basis of all snapshots added so far (randomized range finder, FP64). */
int fast_gpu_ws_build_basis(fast_gpu_ws *ws, double *captured_energy);
/* Full-batch Adam with a cosine learning-rate decay from lr; loss_history
 * [epochs] (mean squared error in scaled units) may be NULL. */
int fast_gpu_ws_train(fast_gpu_ws *ws, int32_t epochs, float lr, float *loss_history);
/* fast_gpu_nr_predictor: user = the fast_gpu_ws.  Returns 0 with d_u_pred
 * written, or non-zero (no prediction) before training.  Stream-ordered
 * device work only (no host synchronisation).  The network's start (or, with
 * use_network = 0, the secant start) is refined by galerkin_iters reduced
 * Newton corrections in the POD basis,
 *   a += (Phi^T K Phi)^-1 Phi^T (f - g(u)),  u = u_start + Phi a,
 * with K the context's last assembled tangent; a correction is skipped when
 * |Phi^T r| <= galerkin_tol |Phi^T f| or Phi^T K Phi is not positive definite
 * (POD-Galerkin projection of the step's equilibrium). */
int fast_gpu_ws_predict(void *ws, int32_t step, double lambda, const double *d_u_last, const double *d_u_prev,
                        const double *d_f, double *d_u_pred);
/* Defaults: use_network 1, galerkin_iters 0, galerkin_tol 1e-3. */
int fast_gpu_ws_configure(fast_gpu_ws *ws, int32_t use_network, int32_t galerkin_iters, double galerkin_tol);
int fast_gpu_ws_report(fast_gpu_ws *ws, fast_gpu_ws_stats *rep);
/* Phi, host [num_eq][modes] row-major. */
int fast_gpu_ws_get_basis(fast_gpu_ws *ws, double *phi);
/* Training inputs [samples][input_dim] and targets [samples][modes] (scaled),
 * as built by fast_gpu_ws_train; either may be NULL. */
int fast_gpu_ws_get_samples(fast_gpu_ws *ws, float *x, float *t);
/* The network input [input_dim] of the last fast_gpu_ws_predict. */
int fast_gpu_ws_last_input(fast_gpu_ws *ws, float *x);

/* The network alone (gradient checks against a CPU oracle).  Parameters are
 * FP32, per layer W [out][in] row-major then b [out].  A batch of one row
 * runs the single-CTA CUDA-core forward fast_gpu_ws_predict uses (the same
 * BF16 operands and FP32 sums in another order); larger batches run the
 * tcgen05 GEMMs of training. */
int fast_gpu_mlp_params(fast_gpu_ws *ws, float *get, const float *set, int64_t *count);
int fast_gpu_mlp_forward(fast_gpu_ws *ws, int32_t batch, const float *x, float *y);
/* Mean squared error against t and its gradient with respect to every parameter. */
int fast_gpu_mlp_loss_grad(fast_gpu_ws *ws, int32_t batch, const float *x, const float *t, float *loss,
                           float *grad);
/* The tensor-core GEMM by itself (host buffers): C[M][N] = sum_k opA(m,k) opB(n,k),
 * opA(m,k) = ta ? A[k*M+m] : A[m*K+k], opB(n,k) = tb ? B[k*N+n] : B[n*K+k];
 * FP32 in and out, BF16 products, FP32 accumulation (split over K across
 * CTAs, partials summed in a fixed order, when there are few output tiles). */
int fast_gpu_mlp_gemm(fast_gpu_ctx *ctx, int32_t M, int32_t N, int32_t K, const float *A, int32_t ta,
                      const float *B, int32_t tb, float *C);

/* ---- linear Newmark time integration -----------------------------------
 * cCtrlNewmark::Solver (ctrl/ctrlnewmark.cpp:79-254) without damping, under
 * the step load q (the same external load at every time, t = 0 included):
 * M a(0) = q, K_eff = K + M/(beta dt^2), per step the effective load
 * q + M (a0 u + a2 v + a3 a), a solve with K_eff and the reference's update
 * of a and v.  Each solve is a PCG (opts->lin, warm-started from the last
 * displacements when lin.warm_start) where the reference factors K_eff
 * once.  Needs densities on the buckets.  Leaves K_eff in the stiffness
 * slot (the next fast_gpu_assemble rebuilds K). */
typedef struct {
  int32_t steps;              /* MAXIMUM.STEPS                                        */
  int32_t damping;            /* 1: RAYLEIGH.DAMPING with omega1, omega2, xi1, xi2     */
  double  dt;                 /* TIME.STEP                                            */
  double  gamma, beta;        /* NEWMARK.PARAMETERS (0.5, 0.25: average acceleration) */
  fast_gpu_solve_opts lin;    /* the step solves                                      */
  fast_gpu_solve_opts mass;   /* M a(0) = q                                           */
  double  omega1, omega2, xi1, xi2;  /* %HEADER.ANALYSIS.RAYLEIGH.DAMPING: C = alpha M + beta K with
                                        cCtrlNewmark::DampingMatrix's alpha, beta
                                        (ctrl/ctrlnewmark.cpp:262-278)                */
} fast_gpu_newmark_opts;

typedef struct {
  int32_t steps_done, failed_step;
  int32_t linear_iterations, max_step_iterations;
  int32_t mass_iterations, escalated_steps;
  double  umax, vmax, amax;   /* max over the steps of the inf-norms (the reference's printout) */
} fast_gpu_newmark_report;

/* q host [num_eq]; u_out, v_out, a_out [num_eq] (final state) may be NULL;
 * probe_hist [steps][nprobe] receives u at the equations probe_eq[k]. */
int fast_gpu_newmark(fast_gpu_ctx *ctx, const double *q, const fast_gpu_newmark_opts *opts, double *u_out,
                     double *v_out, double *a_out, int32_t nprobe, const int32_t *probe_eq, double *probe_hist,
                     fast_gpu_newmark_report *rep);

/* ---- many independent problems -----------------------------------------
 * Each problem is what one FAST run of cLinStat (ctrl/ctrllins.cpp:46-99)
 * solves; their meshes are uploaded together as one mesh whose problem k owns
 * the nodes [node_offsets[k], node_offsets[k+1]) (no element may couple two
 * problems: checked).  Assembly then covers all problems in one pass, and
 * fast_gpu_solve_batch solves every problem to its own PCGSolver stopping test
 * (mlib/sysmat.cpp:1061-1125: |r_k|/|f_k| < tol, |f_k| > 1e11 replaced by 1,
 * u_k = 0 when |f_k| < tol) in one launch, one CTA per problem. */
typedef struct {
  int32_t converged;
  int32_t iterations;
  double  rel_residual;   /* recurrence |r_k|/|f_k| at exit */
} fast_gpu_problem_report;

int fast_gpu_set_problems(fast_gpu_ctx *ctx, int32_t num_problems, const int64_t *node_offsets);
/* f, u host [num_eq]; FP64 only; reps [num_problems] may be NULL.  Returns
 * FAST_GPU_ENONCONV when any problem did not converge. */
int fast_gpu_solve_batch(fast_gpu_ctx *ctx, const double *f, double *u, const fast_gpu_solve_opts *opts,
                         fast_gpu_problem_report *reps);

/* ---- cSysMatrix replacement (mlib/sysmat.h:60-99) ------------------------ */
/* cSysMatrix::Zero */
int fast_gpu_zero(fast_gpu_ctx *ctx, int32_t what);
/* cControl::StiffnessMatrix / MassMatrix over every bucket: element
 * integration (cElmParam::StiffMat elc/elmparam.cpp:539-597, MassMat :672-739)
 * and colour-scheduled scatter (cElement::AddGlobMat elc/element.cpp:2975-3002).
 * Zeroes the target first.  Deterministic: the result is bit-identical run to run. */
int fast_gpu_assemble(fast_gpu_ctx *ctx, int32_t what);
/* cSysMatrix::Add(i, j, v): adds v to K(i,j) and K(j,i) when i != j, like the
 * reference's symmetric matrices; (i, j) must lie in the pattern. */
int fast_gpu_add(fast_gpu_ctx *ctx, int32_t what, int32_t i, int32_t j, double v);
/* cSysMatrix::AddMat(a, M) (mlib/sysmat.h:98, used by cCtrlNewmark for
 * K_eff = K + a0 M, ctrl/ctrlnewmark.cpp:141,160): K += a M over the shared
 * block pattern, on the device.  dst must be FAST_ASM_STIFFNESS and src
 * FAST_ASM_MASS, both assembled (FAST_GPU_ESTATE otherwise).  Fixed DOFs keep
 * the stiffness slot's unit diagonal (the mass slot holds 0 there).  The
 * stiffness slot then holds K + a M: the next stiffness assembly rebuilds K. */
int fast_gpu_add_mat(fast_gpu_ctx *ctx, int32_t dst, double a, int32_t src);
/* cSysMatrix::Get(i, j) */
int fast_gpu_get(fast_gpu_ctx *ctx, int32_t what, int32_t i, int32_t j, double *v);
/* cSysMatrix::MultVect(in, out): out = K in, equation space, host buffers. */
int fast_gpu_mult_vect(fast_gpu_ctx *ctx, int32_t what, const double *x, double *y);
/* cSysMatrix::Solve(b, x) (mlib/sysmat.cpp:966-970 -> PCGSolver :1061-1125):
 * host f and u of length num_eq. */
int fast_gpu_solve(fast_gpu_ctx *ctx, const double *f, double *u,
                   const fast_gpu_solve_opts *opts, fast_gpu_solve_report *rep);
/* Same with device pointers (equation space, length num_eq). */
int fast_gpu_solve_device(fast_gpu_ctx *ctx, const double *d_f, double *d_u,
                          const fast_gpu_solve_opts *opts, fast_gpu_solve_report *rep);

/* ---- external load (host) ---------------------------------------------
 * cControl::ExtLoadVector (ctrl/ctrl.cpp:668-715) for uniform face tractions
 * (%LOAD.CASE.AREA.UNIFORM; cElemLoad::ExtForce load/load.cpp:618-706):
 * face_nodes [num_faces][nodes_per_face] in the Q4 (4) / Q8 (8) face-shape
 * order of cShapeBrick8/20::GetFace (shp/shpsolid.cpp:264-276, 459-471);
 * q [num_faces][3]; local [num_faces] (NULL = all global); f [num_eq] out.
 * Needs no context and no device. */
int fast_gpu_face_load_vector(int64_t num_nodes, const double *coords, const int32_t *node_eq, int32_t num_eq,
                              int32_t num_faces, int32_t nodes_per_face, const int32_t *face_nodes,
                              const double *q, const int32_t *local, int32_t ngp1d, double *f);

/* The same load on the device, from the context's current coordinates (so a
 * fast_gpu_update_coords is followed): fast_gpu_set_face_loads stores the
 * faces once per load case (same arguments as above, node indices of the
 * uploaded mesh); fast_gpu_face_load_device writes scale * f into d_f
 * (device, num_eq).  Every face is integrated by one thread, then each loaded
 * node sums its faces' contributions in face order, so f is bit-identical run
 * to run. */
int fast_gpu_set_face_loads(fast_gpu_ctx *ctx, int32_t num_faces, int32_t nodes_per_face, const int32_t *face_nodes,
                            const double *q, const int32_t *local, int32_t ngp1d);
int fast_gpu_face_load_device(fast_gpu_ctx *ctx, double scale, double *d_f);

/* Support reactions at the current displacements (cControl::SuppReactions,
 * ctrl/ctrl.cpp:844-882): the internal force of every element with a
 * supported node (device) added to all its nodes in element order, minus the
 * face loads with a supported node (same arguments as
 * fast_gpu_face_load_vector) and the nodal loads nodal_f [num_nodes][3] (may
 * be NULL) on supported nodes, both scaled by load_factor.  supported
 * [num_nodes] (NULL: every node with a DOF without an equation).  R
 * [num_nodes][3] out (host); the rows of supported nodes are the reactions. */
int fast_gpu_support_reactions(fast_gpu_ctx *ctx, const uint8_t *supported, int32_t num_faces,
                               int32_t nodes_per_face, const int32_t *face_nodes, const double *q,
                               const int32_t *local, int32_t ngp1d, const double *nodal_f, double load_factor,
                               double *R);

/* ---- stress recovery ----------------------------------------------------
 * Gauss-point strains and stresses at the current displacements
 * (fast_gpu_set_displacement): cElmParam::IntPntStress (elc/elmparam.cpp:
 * 859-935) for elements first .. first+count-1 of a small-strain hex or
 * B-spline bucket,
 * in the caller's element order; strain and stress are host arrays
 * [count][points][6], Voigt xx yy zz xy xz yz (engineering shears), points in
 * the Gauss rule's order (r fastest). */
int fast_gpu_gauss_stress(fast_gpu_ctx *ctx, int32_t bucket, int64_t first, int64_t count, double *strain,
                          double *stress);
/* The printing step's nodal stresses at the current displacements, for a
 * whole small-strain hex or B-spline bucket (B-spline: the same Gauss rule in
 * every direction): elem_nodal [num_elems][nn][6] (caller's element order) =
 * TR x the Gauss-point stresses, TR the extrapolation of
 * cElmParam::CompTRMatrix (elc/elmparam.cpp:1444-1535: least-squares linear
 * field in r, s, t evaluated at the nodes' natural coordinates, for a
 * B-spline element the uniform grid of its control points over [-1, 1]^3,
 * cShapeBspSolid::NodeNatCoord shp/shpbsp.cpp:906-923; the average for a
 * one-point rule),
 * as cElmParam::NodalStress returns them (:1304-1312); nodal [num_nodes][6]
 * their average at each node over the bucket's elements, summed in element
 * order as cControl::PrintAvrNodalStress does (ctrl/ctrl.cpp:2397-2440),
 * 0 at nodes of no element.  Either output may be NULL. */
int fast_gpu_nodal_stress(fast_gpu_ctx *ctx, int32_t bucket, double *elem_nodal, double *nodal);

/* ---- parity / inspection ---------------------------------------------- */
/* Host-only: builds the node-block pattern and element colouring of a mesh
 * without a device and reports them.  rowptr [num_nodes+1], col [nnz_blocks]
 * and color [num_elems of bucket 0] may be NULL (call once with NULLs to get
 * the sizes). */
int fast_gpu_inspect_pattern(const fast_gpu_mesh *mesh, int64_t *nnz_blocks, int64_t *nnz_lower_eq,
                             int32_t *num_colors, int32_t *rowptr, int32_t *col, int32_t *color);
/* Equation-space lower triangle of the assembled matrix as CSR (what the
 * reference's symmetric matrices store).  Call with col == NULL to get nnz.
 * what = FAST_ASM_STIFFNESS_TF32 reads the tensor-core FP32 stiffness. */
int fast_gpu_get_lower_csr(fast_gpu_ctx *ctx, int32_t what, int64_t *nnz,
                           int64_t *rowptr, int32_t *col, double *val);
/* Element matrices of elements [first, first+count) of a bucket, computed by
 * the same device kernels as the assembly: [count][3nn][3nn] row-major in
 * FAST's element DOF order (cElement::GetElmDofs); with
 * FAST_ASM_INTERNAL_FORCE the element internal forces, [count][3nn]; with
 * FAST_ASM_STIFFNESS_TF32 the tensor-core (three-part TF32) element stiffness. */
int fast_gpu_element_matrices(fast_gpu_ctx *ctx, int32_t what, int32_t bucket, int64_t first,
                              int64_t count, double *Ke);

/* ---- measurement ------------------------------------------------------ */
#define FAST_KERNEL_SPMV_FP64  0   /* K.p with FP64 values (FP64 PCG, FP64 residuals)       */
#define FAST_KERNEL_SPMV_FP32  1   /* K.p with FP32 values (mixed path)                     */
#define FAST_KERNEL_ASSEMBLE   2   /* one stiffness assembly (zero fill unless first-touch, all colours) */
#define FAST_KERNEL_PREDICT_NET       3  /* learned predictor: projections, network, start */
#define FAST_KERNEL_PREDICT_GALERKIN  4  /* learned predictor: reduced Newton corrections  */
#define FAST_KERNEL_INTERNAL_FORCE    5  /* one internal-force evaluation                  */
#define FAST_KERNEL_LINEAR_SOLVE      6  /* one fast_gpu_solve_device call                 */
#define FAST_KERNEL_ASSEMBLE_TF32     7  /* one tensor-core stiffness assembly (FP32 blocks)   */
/* Kernels this context has launched so far (every entry point counts). */
int fast_gpu_launch_count(fast_gpu_ctx *ctx, int64_t *count);
/* Live timing: while enabled, every SpMV launched by a solve, every
 * stiffness assembly and each FAST_KERNEL_* span above is bracketed by CUDA
 * events on the context's stream (spans nest).  Enabling resets the
 * statistics. */
int fast_gpu_kernel_timing(fast_gpu_ctx *ctx, int32_t enable);
/* Launches, summed device time and algorithmic bytes per launch (the
 * roofline numerator; 0 for the spans 3-6) of one timed kind since timing
 * was enabled. */
int fast_gpu_kernel_stats(fast_gpu_ctx *ctx, int32_t which, int64_t *launches, double *total_ms,
                          double *bytes_per_launch);

/* ---- solve without device allocation ----------------------------------
 * No counterpart in the reference.  For callers that cannot let a library
 * allocate device memory (their own memory pool owns the device, or a
 * cudaMalloc/cudaFree, which synchronises the device, would stall their other
 * streams): FP64 Jacobi PCG, the same iteration and stopping test as
 * fast_gpu_solve with FAST_PREC_FP64 / FAST_PRECOND_JACOBI, on a caller's
 * equation-space CSR matrix (full symmetric storage: d_rowptr [num_eq+1],
 * d_col / d_val [nnz]), load d_f and solution d_u [num_eq], all device
 * memory.  Needs no context.  Work vectors live in a static device array of
 * the library (20 MB on each device that has loaded it, held until exit), so
 * num_eq is limited to 500000; a larger system is rejected with
 * FAST_GPU_ETOOBIG before any CUDA call.
 *   First call on a device: with CUDA's lazy module loading (the default
 *   unless CUDA_MODULE_LOADING=EAGER) the array is loaded onto the device,
 *   and so takes its 20 MB of device memory, during the first call made
 *   there; that call may also synchronise the device, and fails with
 *   FAST_GPU_ECUDA if no device memory is left.  num_eq = 0 (pointers may be
 *   NULL) does only this set-up and returns FAST_GPU_OK: make it before the
 *   caller's pool takes the device and before any stream capture.  Later
 *   calls allocate nothing.
 *   Every call looks up the array's device address with the caller's device
 *   current.  Calls share the array and it keeps the last call's contents
 *   (each call re-initialises what it uses): calls that overlap on the GPU
 *   race.
 *   tol <= 0 gives 1e-5 and maxit <= 0 gives num_eq, cSysMatrix's defaults
 *   (mlib/sysmat.h:76-77).  Runs on cuda_stream (a cudaStream_t, NULL =
 *   legacy default stream) and synchronises it every 32 iterations; rep may
 *   be NULL (its true_rel_residual is not computed here and is set to -1).
 *   Returns FAST_GPU_EINVAL for a row whose diagonal is not stored, zero or
 *   not finite (Jacobi is undefined), and FAST_GPU_ENONCONV when maxit is
 *   reached or on a breakdown (p.Kp not positive or a non-finite value: K is
 *   not positive definite), the latter with rep->iterations below maxit. */
int fast_gpu_pcg_solve_noalloc(int32_t num_eq, const int64_t *d_rowptr, const int32_t *d_col, const double *d_val,
                               const double *d_f, double *d_u, double tol, int32_t maxit, void *cuda_stream,
                               fast_gpu_solve_report *rep);

#ifdef __cplusplus
}
#endif
#endif /* FAST_GPU_H */
