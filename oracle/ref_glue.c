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
 */
#include <petsc.h>
#include <time.h>

#include "ptatin3d.h"
#include "private/ptatin_impl.h"
#include "ptatin3d_stokes.h"
#include "dmda_element_q2p1.h"
#include "stokes_operators.h"
#include "stokes_operators_mf.h"

struct _p_Vec {
  PetscScalar *a;
};

struct _p_DM {
  PetscInt nel, npe;
  PetscInt *elnidx;
  struct _p_Vec coords;
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

int ref_has_avx(void)
{
#if defined(__AVX__)
  return 1;
#else
  return 0;
#endif
}
