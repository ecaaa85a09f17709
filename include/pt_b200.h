/*
 * pt_b200.h -- C ABI of libpt_b200.so, the B200 (sm_100a) implementation of
 * pTatin3D's matrix-free Q2-P1disc Stokes operator hot path.
 *
 * Plain C types only (no CUDA or PETSc types): pointers, sizes, a status code.
 * Streams are passed as `void *` holding a cudaStream_t.  An op starts on a
 * stream of its own; device-pointer (_d) calls are asynchronous on the op's
 * stream, so a caller whose producers/consumers run on another stream hands
 * that stream over with pt_op_set_stream (NULL = the legacy default stream).
 * Every entry point returns pt_status and never exits the process (the
 * reference CUDA back-end calls cudaDeviceReset()+exit on errors,
 * src/stokes_operators_cuda.cu:46-57).
 *
 * One rank's local problem: on one rank the DMDA ghosted local numbering
 * equals the global numbering, so vectors are the reference's local arrays:
 *   velocity  [3*N]   interleaved (u,v,w) per node, node id i + j*X + k*X*Y,
 *                     X = 2*mx+1, Y = 2*my+1   (src/ptatin3d_stokes.c:121-146)
 *   pressure  [4*nel] four P1 dofs per element (element e = ei+ej*mx+ek*mx*my)
 *   coords    [3*N]   like velocity
 *   eta       [27*nel] quadrature-point viscosity, element-major, qp index
 *                     a*9+b*3+c (c along xi) -- the QPntVolCoefStokes.eta order
 *                     (include/QPntVolCoefStokes_def.h:41-46)
 *   mask      [3*N]   uint8, nonzero on Dirichlet dofs (BCList, scale 1)
 *
 * Two levels of entry point:
 *  - "SpMVOp" level (pt_a11_apply_*, pt_a11_diag_*, pt_a12_apply_*,
 *    pt_a21_apply_*): the element-loop kernels the reference dispatches
 *    through MatA11MF->SpMVOp_MatMult (include/stokes_operators.h:61), i.e.
 *    MFStokesWrapper_A11_{Tensor,AVX,CUDA}, MFStokesWrapper_diagA11,
 *    MFStokesWrapper_A12(_AVX), MFStokesWrapper_A21.  Input already has
 *    Dirichlet entries zeroed by the caller; output is the unassembled local
 *    sum with no BC row treatment.  Output is overwritten (the reference
 *    caller zeroes Yu first, src/stokes_operators.c:1195-1196, so overwrite
 *    and accumulate agree).
 *  - "MatShell" level (pt_matmult_*, pt_getdiag_*): the BC semantics of
 *    MatMult_MFStokes_A11 / MatGetDiagonal_MFStokes_A11 / MatMult_MFStokes_A12 /
 *    MatMult_MFStokes_A21 (src/stokes_operators.c:1156-1222, 1072-1113,
 *    1301-1370, 1444-1509) for one rank, using the mask set with
 *    pt_op_set_bc_mask.
 *
 * Suffixes: _h = host pointers (the call copies in, computes, copies out and
 * synchronises); _d = device pointers, asynchronous on the op's stream.
 */
#ifndef PT_B200_H
#define PT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  PT_OK = 0,
  PT_ERR_BAD_ARG = 1,    /* invalid size, NULL pointer, unknown name */
  PT_ERR_OOM = 2,        /* device allocation failed */
  PT_ERR_CUDA = 3,       /* a CUDA runtime call failed; see pt_last_error() */
  PT_ERR_TIMEOUT = 4,    /* a bounded device-side wait gave up */
  PT_ERR_STATE = 5,      /* coords / eta / mask not set before an apply */
  PT_ERR_UNSUPPORTED = 6 /* valid request this build does not implement */
} pt_status;

typedef struct {
  int32_t mx, my, mz; /* Q2 elements per axis of this rank (>= 1 each) */
  int32_t nx, ny, nz; /* ghosted local node box; 0 = 2*m+1 (the one-rank box) */
  int32_t ox, oy, oz; /* node offset of element (0,0,0) in that box: esi-gsi,
                         esj-gsj, esk-gsk of dmda_element_q2p1.c:395-400 */
} pt_mesh_desc;

typedef struct pt_op pt_op;

/* Human-readable text of the last error on this thread ("" if none). */
const char *pt_last_error(void);
/* Library version string. */
const char *pt_version(void);

/* Operator context.  Replaces MatA11MFCreate/MatA11MFSetup + the back-end
 * SpMVOp_SetUp (src/stokes_operators.c:104-160, 230-279;
 * src/stokes_operators_cuda.cu:243-323).  Allocates device storage for the
 * mesh data; vectors passed to _h calls are staged through op-owned buffers. */
pt_status pt_op_create(const pt_mesh_desc *desc, pt_op **op);
/* Replaces SpMVOp_Destroy (MFA11Destroy_CUDA, src/stokes_operators_cuda.cu:300-323). */
pt_status pt_op_destroy(pt_op *op);
/* Stream for all subsequent work of this op (cudaStream_t as void*; NULL =
 * the legacy default stream).  Waits for the op's previous stream first. */
pt_status pt_op_set_stream(pt_op *op, void *stream);
pt_status pt_op_get_sizes(const pt_op *op, int64_t *nvel, int64_t *npres, int64_t *nel);

/* Mesh data.  Replaces the coordinate / QPntVolCoefStokes uploads of
 * CopyTo_A11_CUDA (src/stokes_operators_cuda.cu:325-431), done here once per
 * change of the data (the reference re-uploads on PetscObjectState change). */
pt_status pt_op_set_coords_h(pt_op *op, const double *coords);
pt_status pt_op_set_coords_d(pt_op *op, const double *coords);
pt_status pt_op_set_eta_h(pt_op *op, const double *eta);
pt_status pt_op_set_eta_d(pt_op *op, const double *eta);
/* eta read with a stride (in doubles) between quadrature points: the reference
 * keeps eta inside the 48-byte QPntVolCoefStokes record, so &qp[0].eta with
 * stride 6 uploads it without a host-side copy by the caller. */
pt_status pt_op_set_eta_strided_h(pt_op *op, const double *eta0, int64_t stride);
pt_status pt_op_set_bc_mask_h(pt_op *op, const uint8_t *mask); /* NULL = no Dirichlet dofs */

/* ---- SpMVOp level ------------------------------------------------------ */

/* y = A11 u (unassembled local).  Replaces MFStokesWrapper_A11_{Tensor,AVX,CUDA}
 * (src/stokes_operators_tensor.c:181-286, src/stokes_operators_avx.c:206-312,
 * src/stokes_operators_cuda.cu:457-532). */
pt_status pt_a11_apply_h(pt_op *op, const double *u, double *y);
pt_status pt_a11_apply_d(pt_op *op, const double *u, double *y);
/* Single-precision apply (FP32 arithmetic and accumulation) for smoothers. */
pt_status pt_a11_apply_f32_d(pt_op *op, const float *u, float *y);

/* d = diag(A11) (unassembled local).  Replaces MFStokesWrapper_diagA11
 * (src/stokes_operators_mf.c:71-135). */
pt_status pt_a11_diag_h(pt_op *op, double *d);
pt_status pt_a11_diag_d(pt_op *op, double *d);

/* yp = B u (divergence, A21).  Replaces MFStokesWrapper_A21
 * (src/stokes_operators_mf.c:862-937). */
pt_status pt_a21_apply_h(pt_op *op, const double *u, double *yp);
pt_status pt_a21_apply_d(pt_op *op, const double *u, double *yp);

/* yu = B^T p (gradient, A12).  Replaces MFStokesWrapper_A12_AVX / MFStokesWrapper_A12
 * (src/stokes_operators_avx.c:682-829, src/stokes_operators_mf.c:792-860). */
pt_status pt_a12_apply_h(pt_op *op, const double *p, double *yu);
pt_status pt_a12_apply_d(pt_op *op, const double *p, double *yu);

/* y = A11 u (SpMVOp level) with no device allocation.  No counterpart in the
 * reference: it is for callers that cannot allocate device memory when they
 * need the operator -- applications that give the whole GPU to their own
 * fixed-size memory pool, processes under a hard device-memory cap that is
 * already used up, or latency-critical paths that must not take
 * cudaMalloc/cudaFree's device-wide synchronisation.  coords, eta, u and y are
 * caller-owned device arrays of a one-rank box (desc->nx..oz zero); the
 * Gauss-point geometry is recomputed into a fixed 16 MiB scratch area that
 * every GPU loading the library holds until exit, so the mesh must satisfy
 * my*mz*243*MXP <= 2^21 (MXP = mx rounded up to 32, 64 or a multiple of 128;
 * a 16x16x16 box fits) or the call returns PT_ERR_BAD_ARG.  The first call on
 * a device looks up the scratch address (cudaGetSymbolAddress) and should come
 * before any stream capture.  All calls share the scratch: calls that overlap
 * on the GPU race.  The call synchronises `stream` (a cudaStream_t, NULL = the
 * legacy default stream) to check the geometry, and returns PT_ERR_BAD_ARG if
 * some w*eta/detJ <= 0. */
pt_status pt_a11_apply_noalloc_d(const pt_mesh_desc *desc, const double *coords, const double *eta,
                                 const double *u, double *y, void *stream);

/* ---- MatShell level (BC semantics, one rank) -------------------------- */

/* y = A11 x with Dirichlet columns zeroed and rows y_k = x_k
 * (MatMult_MFStokes_A11, src/stokes_operators.c:1156-1222). */
pt_status pt_matmult_a11_h(pt_op *op, const double *x, double *y);
pt_status pt_matmult_a11_d(pt_op *op, const double *x, double *y);
pt_status pt_matmult_a11_f32_d(pt_op *op, const float *x, float *y);
/* diag(A11) with Dirichlet slots set to 1 (MatGetDiagonal_MFStokes_A11,
 * src/stokes_operators.c:1072-1113). */
pt_status pt_getdiag_a11_h(pt_op *op, double *d);
pt_status pt_getdiag_a11_d(pt_op *op, double *d);
/* yu = B^T p with Dirichlet rows zeroed (MatMult_MFStokes_A12,
 * src/stokes_operators.c:1301-1370). */
pt_status pt_matmult_a12_h(pt_op *op, const double *p, double *yu);
pt_status pt_matmult_a12_d(pt_op *op, const double *p, double *yu);
/* yp = B u with Dirichlet columns of u zeroed (MatMult_MFStokes_A21,
 * src/stokes_operators.c:1444-1509). */
pt_status pt_matmult_a21_h(pt_op *op, const double *u, double *yp);
pt_status pt_matmult_a21_d(pt_op *op, const double *u, double *yp);

/* ---- Krylov solve of A11 u = f (precision and serving forms) ------------
 *
 * The reference solves the viscous block with FGMRES and multigrid whose
 * smoothers are Chebyshev-Jacobi sweeps on the A11 shell
 * (src/ptatin_driver_linear_ts.c:559-883; PETSc KSPFGMRES, KSPCHEBYSHEV +
 * PCJACOBI, eigenvalue window "esteig 0,0.2,0,1.1").  This solves on the fine
 * level: FP64 outer Krylov (FGMRES or flexible CG) with the FP64
 * MatShell-level A11, preconditioned by Chebyshev on D^-1 A (D =
 * MatGetDiagonal) over [emin, emax] * lambda_max(D^-1 A), optionally in FP32
 * (FP32 vectors, FP32 A11 apply, FP32 D^-1). Dot products are FP64 and
 * deterministic.  The rhs should be zero on Dirichlet dofs.
 *
 * PT_PC_MG is the reference's preconditioner structure: a geometric V-cycle
 * over nested Q2 levels (coordinates injected as DMDARestrictCoordinates-
 * Hierarchy does, Gauss-point eta projected, A11 re-discretised on each level
 * with these kernels, src/ptatin_driver_linear_ts.c:482-514, 674-712), Q2
 * interpolation / its transpose between levels, Chebyshev(cheby_degree)-Jacobi
 * pre- and post-smoothing (FP32 when cheby_fp32) and mg_coarse_degree
 * Chebyshev steps on the coarsest level. */
typedef enum { PT_KSP_FGMRES = 0, PT_KSP_FCG = 1 } pt_ksp_type;
typedef enum { PT_PC_NONE = 0, PT_PC_JACOBI = 1, PT_PC_CHEBY_JACOBI = 2, PT_PC_MG = 3 } pt_pc_type;

typedef struct {
  int32_t ksp;          /* pt_ksp_type */
  int32_t restart;      /* FGMRES restart length */
  int32_t max_it;       /* outer iterations */
  double rtol, atol;    /* ||b - A x|| <= max(rtol ||b - A x0||, atol) */
  int32_t pc;           /* pt_pc_type */
  int32_t cheby_degree; /* Chebyshev steps per application (degree-1 A11 applies) */
  int32_t cheby_fp32;   /* 1: the Chebyshev-Jacobi smoother runs in FP32 */
  double cheby_emin, cheby_emax; /* window, fractions of lambda_max(D^-1 A) */
  int32_t eig_its;      /* Jacobi-PCG (Lanczos) steps for lambda_max */
  int32_t mg_levels;    /* PT_PC_MG: levels (0 = coarsen while every axis is even and >= 4) */
  int32_t mg_coarse_degree; /* PT_PC_MG: Chebyshev steps on the coarsest level */
  int32_t pc_graph;     /* PT_PC_MG: replay the V-cycle as one captured CUDA graph */
  int32_t mg_assembled; /* PT_PC_MG coarse operators: 0 every level re-discretised and matrix-free;
                           1 re-discretised, levels of <= 32^3 elements on stored element
                           matrices and a coarsest level of <= 1200 dofs solved by a dense
                           inverse; 2 as 1, and every level from the first one of <= 64^3
                           elements down is Galerkin, P^T A P element by element
                           (OP_TYPE_MFGALERKIN then OP_TYPE_GALERKIN,
                           src/ptatin_driver_linear_ts.c:64-380, 713-800) */
  int32_t mg_fine_degree; /* PT_PC_MG: Chebyshev steps on the finest level (0 = cheby_degree) */
  int32_t mg_coarse_half; /* PT_PC_MG with cheby_fp32: Galerkin levels' element matrices kept in FP16, each
                             element scaled by its largest entry, FP32 arithmetic (1, default: half the
                             bytes of an FP32 copy); 0: FP32 copies.  Diagonal and lambda_max always come
                             from the FP64 matrices. */
} pt_solve_opts;

typedef struct {
  int32_t its, converged;
  double rnorm0, rnorm; /* true FP64 residual norms, initial and final */
  double lambda_max;    /* estimate of lambda_max(D^-1 A) */
  int64_t a11_f64, a11_f32; /* A11 applies in each precision */
  double seconds;       /* wall time of the solve */
  int32_t mg_levels;    /* PT_PC_MG: levels in the hierarchy (0 otherwise) */
  int32_t reserved;
  double a11_coarse;    /* PT_PC_MG: coarse-level A11 applies, counted in fine-apply
                           units (each weighted by its elements / fine elements) */
} pt_solve_stats;

typedef struct pt_solver pt_solver;

/* Defaults: FGMRES(30), rtol 1e-8, max_it 10000, Chebyshev(3)-Jacobi in FP32,
 * window [0.2, 1.1], 20 Lanczos steps; multigrid with Galerkin coarse levels
 * (mg_assembled 2). */
void pt_solve_opts_default(pt_solve_opts *opts);
/* Allocates the Krylov workspace on the op's device. */
pt_status pt_solver_create(pt_op *op, const pt_solve_opts *opts, pt_solver **solver);
/* x holds the initial guess on entry and the solution on return (device arrays). */
pt_status pt_solver_solve_d(pt_solver *solver, const double *b, double *x, pt_solve_stats *stats);
/* z = P r with the configured preconditioner (PCApply); sets it up first if
 * needed (PCSetUp, redone after the op's coordinates, viscosity or mask
 * change).  Device arrays, FP64. */
pt_status pt_solver_apply_pc_d(pt_solver *solver, const double *r, double *z);
pt_status pt_solver_destroy(pt_solver *solver);

/* ---- batched A11 over many independent boxes ----------------------------
 *
 * No counterpart in the reference (one operator per rank there).  A work-list
 * over n ops (one-rank boxes, coords and eta set): every (problem, x-tile,
 * row, z-chunk) tile, grouped by colour and tile width; an apply is one launch
 * per non-empty class (at most 8 colours x 3 widths) over the concatenated
 * list, and each problem's result is bitwise what its own apply gives.
 * lz[i] = element layers per z-chunk for problem i (0 = the op's default);
 * the autotuner in pt_b200/batch.py picks it. */
typedef struct pt_batch pt_batch;
pt_status pt_batch_create(int n, pt_op *const *ops, const int32_t *lz, pt_batch **batch);
/* As pt_batch_create with every box tiled tile_x elements wide (32, 64 or
 * 128; 0 = each box's own width).  One width for all boxes puts the whole
 * batch in one class per colour, fewer launches per apply. */
pt_status pt_batch_create_tiled(int n, pt_op *const *ops, const int32_t *lz, int32_t tile_x, pt_batch **batch);
pt_status pt_batch_destroy(pt_batch *batch);
/* Colour-class launches of one apply (a masked apply adds one launch for the
 * Dirichlet rows of every problem). */
int64_t pt_batch_launches_per_apply(const pt_batch *batch);
int64_t pt_batch_tiles(const pt_batch *batch);
/* y_i = A11_i u_i for every problem; u, y are DEVICE arrays of n device
 * pointers; masked != 0 gives the MatShell-level BC semantics. */
pt_status pt_batch_a11_apply_d(pt_batch *batch, const double *const *u, double *const *y, int masked, void *stream);
pt_status pt_batch_a11_apply_f32_d(pt_batch *batch, const float *const *u, float *const *y, int masked, void *stream);

/* ---- serving: continuously batched viscous solves ------------------------
 * No counterpart in the reference (one solve per process there).  A server
 * takes requests (A11 u = f on a one-rank box, mask = Dirichlet dofs, f zero
 * there) as they arrive, admits them in FIFO order while slots and the
 * device-memory budget allow, keeps each request's mesh data and Krylov
 * state on the device, and advances all admitted requests together: one
 * flexible-CG iteration (FP64 residuals and dots, Chebyshev(cheby_degree)-
 * Jacobi preconditioner in FP32 or FP64) is one batched A11 work-list plus a
 * fixed number of chunk-list vector kernels for the whole batch.  Each
 * request's result is bitwise the same alone and in any mix. */
typedef struct {
  int64_t memory_budget_bytes; /* device bytes for admitted requests (default 120 GiB) */
  int32_t max_active;          /* requests iterated together (default 256) */
  int32_t lz;                  /* element layers per z-chunk of the A11 tiles (0: per-box default) */
  int32_t tile_x;              /* A11 tile width for every request (32/64/128; 0: per box; default 64) */
  int32_t cheby_fp32, cheby_degree;
  double cheby_emin, cheby_emax;
  int32_t eig_its;
  double rtol, atol;
  int32_t max_it;
} pt_server_opts;

typedef struct {
  int64_t id;                  /* -1: nothing finished */
  int32_t its, status;         /* status 1 converged, 2 max_it, 3 breakdown */
  int32_t converged, reserved;
  double rnorm0, rnorm;        /* FP64 residual norms (recurrence), initial and final */
  double lambda_max;
  double t_submit, t_admit, t_done; /* seconds on the server clock (pt_server_time) */
} pt_server_result;

typedef struct pt_server pt_server;

void pt_server_opts_default(pt_server_opts *opts);
pt_status pt_server_create(const pt_server_opts *opts, pt_server **server);
pt_status pt_server_destroy(pt_server *server);
/* Seconds since the server was created. */
double pt_server_time(const pt_server *server);
/* Queue a request.  The host arrays (coords 3N, eta 27 nel, mask 3N or NULL,
 * f 3N) must stay valid until the request is admitted; x (3N) receives the
 * solution and must stay valid until pt_server_next_done returns its id. */
pt_status pt_server_submit(pt_server *server, int64_t id, const pt_mesh_desc *desc, const double *coords,
                           const double *eta, const uint8_t *mask, const double *f, double *x);
/* Enqueue `iterations` iterations of the admitted requests, admit queued
 * requests while they run, wait, and retire the finished ones. */
pt_status pt_server_step(pt_server *server, int32_t iterations, int32_t *n_active, int32_t *n_queued);
/* Next finished request (res->id = -1 when none). */
pt_status pt_server_next_done(pt_server *server, pt_server_result *res);
pt_status pt_server_stats(const pt_server *server, int64_t *iterations, int64_t *launches, int64_t *bytes_in_use);
/* Host seconds spent enqueueing iterations (incl. batch rebuilds), admitting,
 * waiting for the device, and retiring. */
pt_status pt_server_timers(const pt_server *server, double *enqueue, double *admit, double *wait, double *retire);

/* ---- the whole Stokes operator ------------------------------------------- */

/* Yu = A11 u + A12 p, Yp = A21 u as unassembled local sums, no BCs: replaces
 * MFStokesWrapper_A / MFStokesWrapper_A_AVX (src/stokes_operators_mf.c:711-790,
 * src/stokes_operators_avx.c:439-636).  Yu and Yp are overwritten. */
pt_status pt_stokes_a_apply_d(pt_op *op, const double *u, const double *p, double *yu, double *yp);
pt_status pt_stokes_a_apply_h(pt_op *op, const double *u, const double *p, double *yu, double *yp);
/* MatMult_MFStokes_A (src/stokes_operators.c:893-979) on one rank: Dirichlet
 * columns of xu zeroed, Yu = A11 xu + A12 xp, Yp = A21 xu, then Yu_k = xu_k on
 * Dirichlet dofs (no pressure BCs, no surface constraints). */
pt_status pt_matmult_a_d(pt_op *op, const double *xu, const double *xp, double *yu, double *yp);
pt_status pt_matmult_a_h(pt_op *op, const double *xu, const double *xp, double *yu, double *yp);

/* ---- Gauss-point coefficients from material points --------------------- */

/* Viscosity and density at the Gauss points of the op's elements from
 * material points, the reference's default projection
 * (coefficient_projection_type 1, "Q1"): replaces
 * _SwarmUpdateGaussPropertiesLocalL2ProjectionQ1_MPntPStokes_FineGrid and
 * _SwarmUpdateGaussPropertiesLocalL2ProjectionQ1_MPntPStokes_InterpolateToQuadratePoints
 * (src/material_point_utils.c:1090-1190, 957-1088) on one rank (the
 * cross-rank sum of shared nodes is not included).  Markers: element index
 * wil[n] within the op's element box (MPntStd.wil), local coordinates
 * xi[3n] (MPntStd.xi), eta[n], rho[n] (MPntPStokes).  Outputs eta_qp,
 * rho_qp [27 nel] in QPntVolCoefStokes order (either may be NULL); install != 0
 * also sets eta_qp as the op's viscosity.  Deterministic (no atomics).
 * PT_ERR_BAD_ARG if some wil lies outside the box (those markers are skipped). */
pt_status pt_project_markers_d(pt_op *op, int64_t n, const int32_t *wil, const double *xi, const double *eta,
                               const double *rho, double *eta_qp, double *rho_qp, int install);
pt_status pt_project_markers_h(pt_op *op, int64_t n, const int32_t *wil, const double *xi, const double *eta,
                               const double *rho, double *eta_qp, double *rho_qp, int install);

/* ---- momentum residual ------------------------------------------------------ */

/* Gauss-point body force QPntVolCoefStokes.Fu (include/QPntVolCoefStokes_def.h:
 * 41-46), [27 nel][3] in the viscosity's element-major, point-minor order.
 * The strided form reads three consecutive doubles per record, records
 * `stride` doubles apart: &qp[0].Fu[0] with stride 6 for the reference's
 * 48-byte records. */
pt_status pt_op_set_body_force_h(pt_op *op, const double *fu);
pt_status pt_op_set_body_force_d(pt_op *op, const double *fu);
pt_status pt_op_set_body_force_strided_h(pt_op *op, const double *fu0, int64_t stride);
/* Replaces FormFunctionLocal_U (src/stokes_form_function.c:99-243): the
 * unassembled local momentum residual ru = A11 u + A12 p - F, where F[n,l] =
 * sum_q w detJ N_n(q) Fu_l(q) is the body-force load.  u is the ghosted local
 * velocity as given (the caller has inserted the Dirichlet values,
 * BCListInsertLocal; no column is zeroed), p the element-local pressure; the
 * caller does the local-to-global ADD and BCListResidualDirichlet, as
 * FormFunction_Stokes (:478-580) does.  ru is overwritten.  The load vector F
 * is formed on first use after the coordinates or the body force change. */
pt_status pt_residual_u_d(pt_op *op, const double *u, const double *p, double *ru);
pt_status pt_residual_u_h(pt_op *op, const double *u, const double *p, double *ru);

/* ---- selection, in the style of -a11_op --------------------------------- */

/* Select the A11 kernel by name, like the reference's -a11_op function list
 * (src/stokes_operators.c:123-154).  Names: "b200" (default: stored element
 * matrices for one-rank boxes of at most 32768 elements, the streaming kernel
 * above), "b200_stream" (the streaming kernel with precomputed Gauss-point
 * geometry), "b200_ebe" (stored 81x81 element matrices, element GEMV + node
 * gather; one-rank boxes) and "b200_colour" (8-colour element kernel).  The getter returns the kernel in use.  Unknown names give
 * PT_ERR_BAD_ARG, as the reference's SETERRQ1 "No -a11_op %s". */
pt_status pt_op_set_a11_kernel(pt_op *op, const char *name);
const char *pt_op_get_a11_kernel(const pt_op *op);
/* Tile schedule of the streaming kernel: element layers per z-chunk of a CTA
 * (0 = the default, about 2048 tiles).  Changes the summation order, so
 * results differ in the last bits between schedules (each is deterministic).
 * No counterpart in the reference; set by the autotuner. */
pt_status pt_op_set_tiling(pt_op *op, int32_t lz);
int32_t pt_op_get_tiling(const pt_op *op);

/* Device-side timing helpers: launch count of this library's kernels on this
 * op since the last reset (for benchmark accounting). */
int64_t pt_op_launch_count(const pt_op *op);
void pt_op_reset_launch_count(pt_op *op);

#ifdef __cplusplus
}
#endif
#endif
