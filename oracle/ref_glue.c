/*
 * Route-A glue: lets the reference's own operator sources
 *   src/stokes_operators_tensor.c, src/stokes_operators_avx.c,
 *   src/stokes_operators_mf.c, src/element_utils_q2.c, src/element_utils_q1.c
 * (compiled unmodified from the reference tree by oracle/Makefile) run on plain
 * arrays for one process.  TEST INFRASTRUCTURE ONLY.
 *
 * Everything arithmetic comes from the reference sources.  This file only
 * supplies the PETSc/pTatin data-access routines those sources call, as
 * marshalling over caller-owned arrays:
 *   - DM / Vec accessors: a DM carries the local coordinate array and the
 *     element table; a Vec wraps a pointer.
 *   - DMDAGetElements_pTatinQ2P1: the Q2 table of dmda_element_q2p1.c:395-455
 *     (one rank: esi=gsi=0) and the P1 table of dmda_element_q2p1.c:488-545
 *     (4 consecutive dofs per element).
 *   - element gathers / scatter-adds (dmda_element_q2p1.c:626-671,
 *     ptatin3d_stokes.c:49-70,270-318).
 *   - VolumeQuadratureGet*CellData_Stokes (ptatin3d_stokes.c:453-475) over an
 *     array of QPntVolCoefStokes built from a plain eta[27*nel].
 *   - PetscDTGaussQuadrature for n=3 (PETSc 3.8.3, absent here): closed form
 *     of the Golub-Welsch result, nodes 0, +-sqrt(3/5), weights 8/9, 5/9.
 *   - a PhysCompStokes carrying the quadrature for the momentum residual
 *     FormFunctionLocal_U (src/stokes_form_function.c:99-243);
 *   - for the marker -> Gauss-point viscosity projection of
 *     src/material_point_utils.c: local vectors of a dof-1 Q2 node grid
 *     (DMGetLocalVector ...), local<->global on one rank (identity / add),
 *     VecPointwiseDivide, and the dof-1 element index / add-values helpers
 *     (dmda_element_q2p1.c).
 */
#include <petsc.h>
#include <time.h>

#include "ptatin3d.h"
#include "private/ptatin_impl.h"
#include "ptatin3d_stokes.h"
#include "dmda_element_q2p1.h"
#include "stokes_operators.h"
#include "stokes_operators_mf.h"
#include "MPntStd_def.h"
#include "MPntPStokes_def.h"
#include "material_point_utils.h"
#include "private/ptatin3d_stokes_impl.h"

struct _p_Vec {
  PetscScalar *a;
  PetscInt n;
};

struct _p_DM {
  PetscInt nel, npe;
  PetscInt *elnidx;
  struct _p_Vec coords;
  PetscInt nlocal; /* entries of a local (= global, one rank) vector */
};

PetscErrorCode PetscDTGaussQuadrature(PetscInt n, PetscReal a, PetscReal b, PetscReal *x, PetscReal *w)
{
  const PetscReal s = sqrt(3.0 / 5.0);
  if (n != 3) return PETSC_ERR_SUP;
  x[0] = 0.5 * (a + b) - s * 0.5 * (b - a);
  x[1] = 0.5 * (a + b);
  x[2] = 0.5 * (a + b) + s * 0.5 * (b - a);
  w[0] = w[2] = 0.5 * (b - a) * (5.0 / 9.0);
  w[1] = 0.5 * (b - a) * (8.0 / 9.0);
  return 0;
}

PetscErrorCode PetscTime(PetscLogDouble *t)
{
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  *t = (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
  return 0;
}

PetscErrorCode DMGetCoordinateDM(DM dm, DM *cda) { *cda = dm; return 0; }
PetscErrorCode DMGetCoordinatesLocal(DM dm, Vec *v) { *v = &dm->coords; return 0; }
PetscErrorCode VecGetArrayRead(Vec v, const PetscScalar **a) { *a = v->a; return 0; }
PetscErrorCode VecRestoreArrayRead(Vec v, const PetscScalar **a) { (void)v; *a = NULL; return 0; }
PetscErrorCode VecGetArray(Vec v, PetscScalar **a) { *a = v->a; return 0; }
PetscErrorCode VecRestoreArray(Vec v, PetscScalar **a) { (void)v; *a = NULL; return 0; }

PetscErrorCode DMDAGetElements_pTatinQ2P1(DM dm, PetscInt *nel, PetscInt *nen, const PetscInt *e[])
{
  *nel = dm->nel;
  *nen = dm->npe;
  *e = dm->elnidx;
  return 0;
}

PetscErrorCode DMDAGetElementCoordinatesQ2_3D(PetscScalar elcoords[], PetscInt elnid[], PetscScalar LA_gcoords[])
{
  PetscInt n;
  for (n = 0; n < 27; n++) {
    elcoords[3 * n] = LA_gcoords[3 * elnid[n]];
    elcoords[3 * n + 1] = LA_gcoords[3 * elnid[n] + 1];
    elcoords[3 * n + 2] = LA_gcoords[3 * elnid[n] + 2];
  }
  return 0;
}

PetscErrorCode DMDAGetVectorElementFieldQ2_3D(PetscScalar elfield[], PetscInt elnid[], PetscScalar LA_gfield[])
{
  return DMDAGetElementCoordinatesQ2_3D(elfield, elnid, LA_gfield);
}

PetscErrorCode DMDAGetScalarElementField(PetscScalar elfield[], PetscInt npe, PetscInt elnid[], PetscScalar LA_gfield[])
{
  PetscInt n;
  for (n = 0; n < npe; n++) elfield[n] = LA_gfield[elnid[n]];
  return 0;
}

PetscErrorCode StokesVelocity_GetElementLocalIndices(PetscInt idx[], PetscInt elnid[])
{
  PetscInt n;
  for (n = 0; n < 27; n++) {
    idx[3 * n] = 3 * elnid[n];
    idx[3 * n + 1] = 3 * elnid[n] + 1;
    idx[3 * n + 2] = 3 * elnid[n] + 2;
  }
  return 0;
}

PetscErrorCode StokesPressure_GetElementLocalIndices(PetscInt idx[], PetscInt elnid[])
{
  PetscInt n;
  for (n = 0; n < 4; n++) idx[n] = elnid[n];
  return 0;
}

PetscErrorCode DMDASetValuesLocalStencil_AddValues_Stokes_Velocity(PetscScalar *F, PetscInt eqn[], PetscScalar Fe[])
{
  PetscInt n;
  for (n = 0; n < 81; n++) F[eqn[n]] += Fe[n];
  return 0;
}

PetscErrorCode DMDASetValuesLocalStencil_AddValues_Stokes_Pressure(PetscScalar *F, PetscInt eqn[], PetscScalar Fe[])
{
  PetscInt n;
  for (n = 0; n < 4; n++) F[eqn[n]] += Fe[n];
  return 0;
}

PetscErrorCode VolumeQuadratureGetAllCellData_Stokes(Quadrature Q, QPntVolCoefStokes *coeffs[])
{
  *coeffs = (QPntVolCoefStokes *)Q->q_weight; /* the glue parks the coefficient array here */
  return 0;
}

PetscErrorCode VolumeQuadratureGetCellData_Stokes(Quadrature Q, QPntVolCoefStokes coeffs[], PetscInt cidx, QPntVolCoefStokes *cell[])
{
  if (cidx >= Q->n_elements) return PETSC_ERR_ARG_SIZ;
  *cell = &coeffs[cidx * Q->npoints];
  return 0;
}

/* ---- vectors of a dof-1 node grid on one rank (local == global) ---------- */

PetscErrorCode DMGetLocalVector(DM dm, Vec *v)
{
  struct _p_Vec *x = (struct _p_Vec *)calloc(1, sizeof *x);
  if (!x) return PETSC_ERR_MEM;
  x->n = dm->nlocal;
  x->a = (PetscScalar *)calloc((size_t)(x->n > 0 ? x->n : 1), sizeof(PetscScalar));
  if (!x->a) return PETSC_ERR_MEM;
  *v = x;
  return 0;
}

PetscErrorCode DMRestoreLocalVector(DM dm, Vec *v)
{
  (void)dm;
  if (*v) {
    free((*v)->a);
    free(*v);
  }
  *v = NULL;
  return 0;
}

PetscErrorCode VecZeroEntries(Vec v)
{
  memset(v->a, 0, sizeof(PetscScalar) * (size_t)v->n);
  return 0;
}

PetscErrorCode DMLocalToGlobalBegin(DM dm, Vec l, InsertMode mode, Vec g)
{
  PetscInt i;
  (void)dm;
  for (i = 0; i < g->n; i++) g->a[i] = (mode == ADD_VALUES) ? g->a[i] + l->a[i] : l->a[i];
  return 0;
}

PetscErrorCode DMLocalToGlobalEnd(DM dm, Vec l, InsertMode mode, Vec g)
{
  (void)dm; (void)l; (void)mode; (void)g;
  return 0;
}

PetscErrorCode DMGlobalToLocalBegin(DM dm, Vec g, InsertMode mode, Vec l)
{
  PetscInt i;
  (void)dm; (void)mode;
  for (i = 0; i < l->n; i++) l->a[i] = g->a[i];
  return 0;
}

PetscErrorCode DMGlobalToLocalEnd(DM dm, Vec g, InsertMode mode, Vec l)
{
  (void)dm; (void)g; (void)mode; (void)l;
  return 0;
}

PetscErrorCode VecPointwiseDivide(Vec w, Vec x, Vec y)
{
  PetscInt i;
  for (i = 0; i < w->n; i++) w->a[i] = x->a[i] / y->a[i];
  return 0;
}

PetscErrorCode Q2GetElementLocalIndicesDOF(PetscInt el_localIndices[], PetscInt ndof, PetscInt elnid[])
{
  PetscInt n, d;
  for (n = 0; n < 27; n++)
    for (d = 0; d < ndof; d++) el_localIndices[ndof * n + d] = ndof * elnid[n] + d;
  return 0;
}

PetscErrorCode DMDASetValuesLocalStencil_AddValues_DOF(PetscScalar *fields_F, PetscInt ndof, PetscInt eqn[],
                                                       PetscScalar Fe[])
{
  PetscInt n;
  for (n = 0; n < 27 * ndof; n++) fields_F[eqn[n]] += Fe[n];
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Plain-array entry points (ctypes)                                          */
/* ------------------------------------------------------------------------ */

typedef struct {
  struct _p_DM dau, dap;
  struct _p_Quadrature volQ;
  QPntVolCoefStokes *qp;
} RefCtx;

static void q2_table(int mx, int my, int mz, PetscInt *idx)
{
  const PetscInt X = 2 * mx + 1, Y = 2 * my + 1;
  PetscInt ei, ej, ek, a, b, c, e = 0;
  for (ek = 0; ek < mz; ek++)
    for (ej = 0; ej < my; ej++)
      for (ei = 0; ei < mx; ei++) {
        for (a = 0; a < 3; a++)
          for (b = 0; b < 3; b++)
            for (c = 0; c < 3; c++)
              idx[27 * e + 9 * a + 3 * b + c] = (2 * ei + c) + (2 * ej + b) * X + (2 * ek + a) * X * Y;
        e++;
      }
}

static int ctx_init(RefCtx *c, int mx, int my, int mz, const double *coords, const double *eta)
{
  const PetscInt nel = (PetscInt)mx * my * mz;
  PetscInt e;
  memset(c, 0, sizeof *c);
  c->dau.nel = nel; c->dau.npe = 27;
  c->dau.elnidx = (PetscInt *)malloc(sizeof(PetscInt) * 27 * (nel + 1));
  c->dap.nel = nel; c->dap.npe = 4;
  c->dap.elnidx = (PetscInt *)malloc(sizeof(PetscInt) * 4 * (nel + 1));
  c->qp = (QPntVolCoefStokes *)calloc((size_t)27 * (nel + 1), sizeof(QPntVolCoefStokes));
  if (!c->dau.elnidx || !c->dap.elnidx || !c->qp) return 1;
  q2_table(mx, my, mz, c->dau.elnidx);
  for (e = 0; e < 4 * nel; e++) c->dap.elnidx[e] = e;
  if (eta)
    for (e = 0; e < 27 * nel; e++) c->qp[e].eta = eta[e];
  c->dau.coords.a = (PetscScalar *)coords;
  c->dap.coords.a = (PetscScalar *)coords;
  c->volQ.dim = 3;
  c->volQ.npoints = 27;
  c->volQ.n_elements = nel;
  c->volQ.q_weight = (PetscReal *)c->qp;
  return 0;
}

static void ctx_free(RefCtx *c)
{
  free(c->dau.elnidx);
  free(c->dap.elnidx);
  free(c->qp);
}

/* kind: 0 tensor, 1 avx, 2 ref. y += A11 u. */
int ref_a11(int kind, int mx, int my, int mz, const double *coords, const double *eta, double *u, double *y)
{
  RefCtx c;
  int ierr;
  if (ctx_init(&c, mx, my, mz, coords, eta)) return 1;
  if (kind == 0) ierr = MFStokesWrapper_A11_Tensor(NULL, &c.volQ, &c.dau, u, y);
#if defined(__AVX__)
  else if (kind == 1) ierr = MFStokesWrapper_A11_AVX(NULL, &c.volQ, &c.dau, u, y);
#endif
  else if (kind == 2) ierr = MFStokesWrapper_A11(NULL, &c.volQ, &c.dau, u, y);
  else ierr = 2;
  ctx_free(&c);
  return ierr;
}

int ref_diag(int mx, int my, int mz, const double *coords, const double *eta, double *y)
{
  RefCtx c;
  int ierr;
  if (ctx_init(&c, mx, my, mz, coords, eta)) return 1;
  ierr = MFStokesWrapper_diagA11(&c.volQ, &c.dau, y);
  ctx_free(&c);
  return ierr;
}

int ref_a21(int mx, int my, int mz, const double *coords, double *u, double *yp)
{
  RefCtx c;
  int ierr;
  if (ctx_init(&c, mx, my, mz, coords, NULL)) return 1;
  ierr = MFStokesWrapper_A21(&c.volQ, &c.dau, &c.dap, u, yp);
  ctx_free(&c);
  return ierr;
}

/* kind: 1 avx, 2 ref. */
int ref_a12(int kind, int mx, int my, int mz, const double *coords, double *p, double *yu)
{
  RefCtx c;
  int ierr;
  if (ctx_init(&c, mx, my, mz, coords, NULL)) return 1;
#if defined(__AVX__)
  if (kind == 1) ierr = MFStokesWrapper_A12_AVX(&c.volQ, &c.dau, &c.dap, p, yu);
  else
#endif
  if (kind == 2) ierr = MFStokesWrapper_A12(&c.volQ, &c.dau, &c.dap, p, yu);
  else ierr = 2;
  ctx_free(&c);
  return ierr;
}

/* The whole Stokes operator on one rank: Yu = A11 u + A12 p, Yp = A21 u
 * (MFStokesWrapper_A_AVX, src/stokes_operators_avx.c:439-636, kind 1;
 * MFStokesWrapper_A, src/stokes_operators_mf.c:711-790, kind 2). */
int ref_stokes_a(int kind, int mx, int my, int mz, const double *coords, const double *eta, double *u, double *p,
                 double *yu, double *yp)
{
  RefCtx c;
  int ierr;
  if (ctx_init(&c, mx, my, mz, coords, eta)) return 1;
#if defined(__AVX__)
  if (kind == 1) ierr = MFStokesWrapper_A_AVX(&c.volQ, &c.dau, u, &c.dap, p, yu, yp);
  else
#endif
  if (kind == 2) ierr = MFStokesWrapper_A(&c.volQ, &c.dau, u, &c.dap, p, yu, yp);
  else ierr = 2;
  ctx_free(&c);
  return ierr;
}

/* The momentum residual FormFunctionLocal_U (src/stokes_form_function.c:99-243)
 * on one rank: Ru += A11 u + A12 p - (body force), element by element with
 * the reference's own geometry and P1GRel pressure basis; fu[3*q] holds the
 * Gauss-point body force QPntVolCoefStokes.Fu.  u is used as given (the
 * caller inserts the Dirichlet values, BCListInsertLocal). */
PetscErrorCode FormFunctionLocal_U(PhysCompStokes, DM, PetscScalar[], DM, PetscScalar[], PetscScalar[]);

int ref_residual_u(int mx, int my, int mz, const double *coords, const double *eta, const double *fu, double *u,
                   double *p, double *ru)
{
  RefCtx c;
  struct _p_PhysCompStokes stokes;
  PetscInt q;
  int ierr;
  if (ctx_init(&c, mx, my, mz, coords, eta)) return 1;
  for (q = 0; q < 27 * (PetscInt)mx * my * mz; q++) {
    c.qp[q].Fu[0] = fu[3 * q];
    c.qp[q].Fu[1] = fu[3 * q + 1];
    c.qp[q].Fu[2] = fu[3 * q + 2];
  }
  memset(&stokes, 0, sizeof stokes);
  stokes.volQ = &c.volQ;
  ierr = FormFunctionLocal_U(&stokes, &c.dau, u, &c.dap, p, ru);
  ctx_free(&c);
  return ierr;
}

/* Marker -> Gauss-point viscosity and density, the reference's default Q1
 * projection (coefficient_projection_type 1) on one level:
 * _SwarmUpdateGaussPropertiesLocalL2ProjectionQ1_MPntPStokes_FineGrid and
 * _SwarmUpdateGaussPropertiesLocalL2ProjectionQ1_MPntPStokes_InterpolateToQuadratePoints
 * (src/material_point_utils.c:1090-1190, 957-1088).  Markers: element index
 * wil, local coordinates xi[3], eta, rho.  Gauss points: the reference's
 * QuadratureCreateGauss_3pnt_3D table (src/quadrature.c:136-167). */
PetscErrorCode _SwarmUpdateGaussPropertiesLocalL2ProjectionQ1_MPntPStokes_FineGrid(DM, Vec, Vec, Vec, const int,
                                                                                   MPntStd[], MPntPStokes[]);
PetscErrorCode _SwarmUpdateGaussPropertiesLocalL2ProjectionQ1_MPntPStokes_InterpolateToQuadratePoints(
    DM, Vec, Vec, Quadrature, SurfaceQuadrature, MeshFacetInfo);

int ref_marker_project(int mx, int my, int mz, int npoints, const int *wil, const double *xi, const double *eta_p,
                       const double *rho_p, double *eta_qp, double *rho_qp)
{
  RefCtx c;
  int ierr = 0, p, k;
  const double s = 0.774596669241483, xi1[3] = {-0.774596669241483, 0.0, 0.774596669241483};
  PetscReal qxi[81];
  struct _p_Vec A1, A2, B;
  MPntStd *std = NULL;
  MPntPStokes *stk = NULL;
  (void)s;
  if (ctx_init(&c, mx, my, mz, NULL, NULL)) return 1;
  c.dau.nlocal = (PetscInt)(2 * mx + 1) * (2 * my + 1) * (2 * mz + 1);
  for (k = 0; k < 27; k++) {
    qxi[3 * k] = xi1[k % 3];
    qxi[3 * k + 1] = xi1[(k / 3) % 3];
    qxi[3 * k + 2] = xi1[k / 9];
  }
  c.volQ.q_xi_coor = qxi;
  A1.n = A2.n = B.n = c.dau.nlocal;
  A1.a = (PetscScalar *)calloc((size_t)A1.n, sizeof(PetscScalar));
  A2.a = (PetscScalar *)calloc((size_t)A2.n, sizeof(PetscScalar));
  B.a = (PetscScalar *)calloc((size_t)B.n, sizeof(PetscScalar));
  std = (MPntStd *)calloc((size_t)(npoints > 0 ? npoints : 1), sizeof(MPntStd));
  stk = (MPntPStokes *)calloc((size_t)(npoints > 0 ? npoints : 1), sizeof(MPntPStokes));
  if (!A1.a || !A2.a || !B.a || !std || !stk) ierr = 1;
  for (p = 0; !ierr && p < npoints; p++) {
    std[p].pid = p;
    std[p].wil = wil[p];
    std[p].xi[0] = xi[3 * p]; std[p].xi[1] = xi[3 * p + 1]; std[p].xi[2] = xi[3 * p + 2];
    stk[p].eta = eta_p[p];
    stk[p].rho = rho_p[p];
  }
  if (!ierr) ierr = _SwarmUpdateGaussPropertiesLocalL2ProjectionQ1_MPntPStokes_FineGrid(&c.dau, &A1, &A2, &B, npoints,
                                                                                        std, stk);
  if (!ierr)
    ierr = _SwarmUpdateGaussPropertiesLocalL2ProjectionQ1_MPntPStokes_InterpolateToQuadratePoints(&c.dau, &A1, &A2,
                                                                                                  &c.volQ, NULL, NULL);
  if (!ierr)
    for (k = 0; k < 27 * mx * my * mz; k++) {
      eta_qp[k] = c.qp[k].eta;
      rho_qp[k] = c.qp[k].rho;
    }
  free(A1.a); free(A2.a); free(B.a); free(std); free(stk);
  ctx_free(&c);
  return ierr;
}

int ref_has_avx(void)
{
#if defined(__AVX__)
  return 1;
#else
  return 0;
#endif
}

/* OpenMP threads of the reference's CPU operators (the timed baseline reports
 * all host threads and one thread); returns the count now in effect. */
#if defined(_OPENMP)
#include <omp.h>
#endif
int ref_set_threads(int n)
{
#if defined(_OPENMP)
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}
