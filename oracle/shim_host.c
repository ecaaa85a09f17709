/*
 * Runs the PETSc plug-in (ptatin-gene_b200/shim/stokes_operators_b200.c) without
 * PETSc.  TEST INFRASTRUCTURE ONLY: linked with the plug-in and libpt_b200.so
 * into oracle/_ref/libshimtest.so by oracle/Makefile, and driven from
 * tests/test_gpu_shim.py through the shimtest_* entry points below.
 *
 * The plug-in is compiled unmodified against the reference's headers and the
 * PETSc stand-in (ref_stub/).  This file supplies what it calls:
 *   - PETSc objects with a state counter (PetscObjectStateGet), one composed
 *     object slot per name (PetscObjectQuery / Compose), reference-counted
 *     containers with a destroy callback (PetscContainer*);
 *   - a one-rank velocity DM: DMDAGetCornersElementQ2 / DMDAGetGhostCorners
 *     give the element box (0,0,0)+(mx,my,mz) in its node box, or an element
 *     sub-box in a larger ghosted node box (the multi-rank local layout);
 *     DMGetCoordinatesLocal gives a coordinate Vec whose state the test bumps
 *     when it moves the mesh;
 *   - a Quadrature whose QPntVolCoefStokes records
 *     (include/QPntVolCoefStokes_def.h:41-46, eta at offset 0) hold the
 *     viscosity, VolumeQuadratureGetAllCellData_Stokes returning them;
 *   - a MatA11MF (include/stokes_operators.h:48-64) and a Stokes Mat object
 *     whose states version the viscosity.
 */
#include <petsc.h>

#include "ptatin3d.h"
#include "private/ptatin_impl.h"
#include "ptatin3d_stokes.h"
#include "dmda_element_q2p1.h"
#include "stokes_operators.h"

#include "pt_b200.h"

#define MAX_COMPOSED 4

struct _p_PetscObject {
  PetscObjectState state;
  int refct;
  const char *names[MAX_COMPOSED];
  struct _p_PetscObject *composed[MAX_COMPOSED];
};

struct _p_Vec {
  struct _p_PetscObject hdr;
  PetscScalar *a;
  PetscInt n;
};

struct _p_PetscContainer {
  struct _p_PetscObject hdr;
  void *ptr;
  PetscErrorCode (*destroy)(void *);
};

struct _p_DM {
  struct _p_PetscObject hdr;
  PetscInt sei, sej, sek, mx, my, mz; /* element box: first element (global), counts */
  PetscInt gsi, gsj, gsk, X, Y, Z;    /* ghosted node box: first node (global), sizes */
  struct _p_Vec coords;
};

struct _p_Mat {
  struct _p_PetscObject hdr;
};

/* ---- PETSc object routines ------------------------------------------------ */

static void obj_release(struct _p_PetscObject *o);

static void container_release(PetscContainer c)
{
  if (--c->hdr.refct > 0) return;
  if (c->destroy) c->destroy(c->ptr);
  free(c);
}

static void obj_release(struct _p_PetscObject *o)
{
  /* the only composed objects in these tests are containers */
  container_release((PetscContainer)o);
}

PetscErrorCode PetscObjectStateGet(PetscObject o, PetscObjectState *s) { *s = o->state; return 0; }
PetscErrorCode PetscObjectReference(PetscObject o) { o->refct++; return 0; }
MPI_Comm PetscObjectComm(PetscObject o) { (void)o; return PETSC_COMM_SELF; }

PetscErrorCode PetscObjectQuery(PetscObject o, const char name[], PetscObject *out)
{
  int i;
  *out = NULL;
  for (i = 0; i < MAX_COMPOSED; i++)
    if (o->names[i] && !strcmp(o->names[i], name)) *out = o->composed[i];
  return 0;
}

PetscErrorCode PetscObjectCompose(PetscObject o, const char name[], PetscObject x)
{
  int i, slot = -1;
  for (i = 0; i < MAX_COMPOSED; i++)
    if (o->names[i] && !strcmp(o->names[i], name)) slot = i;
  for (i = 0; slot < 0 && i < MAX_COMPOSED; i++)
    if (!o->names[i]) slot = i;
  if (slot < 0) return PETSC_ERR_MEM;
  if (x) x->refct++;
  if (o->composed[slot]) obj_release(o->composed[slot]);
  o->names[slot] = x ? name : NULL;
  o->composed[slot] = x;
  return 0;
}

PetscErrorCode PetscContainerCreate(MPI_Comm comm, PetscContainer *c)
{
  (void)comm;
  *c = (PetscContainer)calloc(1, sizeof(struct _p_PetscContainer));
  if (!*c) return PETSC_ERR_MEM;
  (*c)->hdr.refct = 1;
  return 0;
}
PetscErrorCode PetscContainerSetPointer(PetscContainer c, void *p) { c->ptr = p; return 0; }
PetscErrorCode PetscContainerGetPointer(PetscContainer c, void **p) { *p = c->ptr; return 0; }
PetscErrorCode PetscContainerSetUserDestroy(PetscContainer c, PetscErrorCode (*d)(void *)) { c->destroy = d; return 0; }
PetscErrorCode PetscContainerDestroy(PetscContainer *c)
{
  if (*c) container_release(*c);
  *c = NULL;
  return 0;
}

PetscErrorCode PetscFunctionListAdd_Private(PetscFunctionList *l, const char name[], void (*f)(void))
{
  (void)l; (void)name; (void)f;
  return 0;
}

/* ---- DM, Vec, Quadrature ------------------------------------------------------ */

PetscErrorCode DMDAGetCornersElementQ2(DM da, PetscInt *sei, PetscInt *sej, PetscInt *sek, PetscInt *mx,
                                       PetscInt *my, PetscInt *mz)
{
  *sei = da->sei; *sej = da->sej; *sek = da->sek;
  *mx = da->mx; *my = da->my; *mz = da->mz;
  return 0;
}

PetscErrorCode DMDAGetGhostCorners(DM da, PetscInt *gsi, PetscInt *gsj, PetscInt *gsk, PetscInt *X, PetscInt *Y,
                                   PetscInt *Z)
{
  *gsi = da->gsi; *gsj = da->gsj; *gsk = da->gsk;
  *X = da->X; *Y = da->Y; *Z = da->Z;
  return 0;
}

PetscErrorCode DMGetCoordinatesLocal(DM dm, Vec *v) { *v = &dm->coords; return 0; }
PetscErrorCode VecGetArrayRead(Vec v, const PetscScalar **a) { *a = v->a; return 0; }
PetscErrorCode VecRestoreArrayRead(Vec v, const PetscScalar **a) { (void)v; *a = NULL; return 0; }

PetscErrorCode VolumeQuadratureGetAllCellData_Stokes(Quadrature Q, QPntVolCoefStokes *coeffs[])
{
  *coeffs = (QPntVolCoefStokes *)Q->q_weight; /* parked here by shimtest_create */
  return 0;
}

/* ---- the plug-in's entry points (stokes_operators_b200.c) ------------------- */

PetscErrorCode MFA11SetUp_B200(MatA11MF);
PetscErrorCode MFA11Destroy_B200(MatA11MF);
PetscErrorCode MFStokesWrapper_A11_B200(MatA11MF, Quadrature, DM, PetscScalar[], PetscScalar[]);
PetscErrorCode MFStokesWrapper_diagA11_B200(MatA11MF, Quadrature, DM, PetscScalar[]);
PetscErrorCode MFStokesWrapper_A12_B200(Quadrature, DM, DM, PetscScalar[], PetscScalar[]);
PetscErrorCode MFStokesWrapper_A21_B200(Quadrature, DM, DM, PetscScalar[], PetscScalar[]);
PetscErrorCode MFStokesWrapper_A_B200(Mat, Quadrature, DM, PetscScalar[], DM, PetscScalar[], PetscScalar[],
                                      PetscScalar[]);
PetscErrorCode MFA11B200GetOp(DM, pt_op **);
PetscErrorCode MatA11MFRegister_B200(PetscFunctionList *, PetscFunctionList *, PetscFunctionList *);

/* ---- test entry points ---------------------------------------------------------- */

typedef struct {
  struct _p_DM dau;
  struct _p_Quadrature volQ;
  struct _p_MatA11MF mf;
  struct _p_Mat stokes;
  QPntVolCoefStokes *qp;
  PetscInt nel;
} ShimTest;

/* node box (X,Y,Z) with the element box starting at node offset (ox,oy,oz);
 * X = 0 means the one-rank box 2m+1. */
void *shimtest_create(int mx, int my, int mz, int X, int Y, int Z, int ox, int oy, int oz, double *coords,
                      const double *eta)
{
  ShimTest *t = (ShimTest *)calloc(1, sizeof *t);
  PetscInt e;
  if (!t) return NULL;
  t->nel = (PetscInt)mx * my * mz;
  t->dau.mx = mx; t->dau.my = my; t->dau.mz = mz;
  t->dau.X = X ? X : 2 * mx + 1; t->dau.Y = Y ? Y : 2 * my + 1; t->dau.Z = Z ? Z : 2 * mz + 1;
  /* element (0,0,0)'s first node sits at (ox,oy,oz) of the node box: global
   * starts sei = gsi + ox (one element spans 2 nodes, so sei counts nodes) */
  t->dau.gsi = 10; t->dau.gsj = 20; t->dau.gsk = 30;
  t->dau.sei = t->dau.gsi + ox; t->dau.sej = t->dau.gsj + oy; t->dau.sek = t->dau.gsk + oz;
  t->dau.coords.a = coords;
  t->dau.coords.n = 3 * t->dau.X * t->dau.Y * t->dau.Z;
  t->dau.coords.hdr.state = 1;
  t->qp = (QPntVolCoefStokes *)calloc((size_t)27 * t->nel, sizeof(QPntVolCoefStokes));
  if (!t->qp) { free(t); return NULL; }
  for (e = 0; e < 27 * t->nel; e++) {
    t->qp[e].eta = eta[e];
    t->qp[e].rho = -1.0;        /* the other members are not viscosity: fill them */
    t->qp[e].Fu[0] = t->qp[e].Fu[1] = t->qp[e].Fu[2] = 7.0;
    t->qp[e].Fp = -3.0;
  }
  t->volQ.dim = 3;
  t->volQ.npoints = 27;
  t->volQ.n_elements = t->nel;
  t->volQ.q_weight = (PetscReal *)t->qp;
  t->mf.daUVW = &t->dau;
  t->mf.volQ = &t->volQ;
  t->mf.state = 1;
  t->stokes.hdr.state = 1;
  if (MFA11SetUp_B200(&t->mf)) { free(t->qp); free(t); return NULL; }
  return t;
}

int shimtest_register(void)
{
  PetscFunctionList a = NULL, b = NULL, c = NULL;
  return MatA11MFRegister_B200(&a, &b, &c);
}

int shimtest_a11(void *h, double *u, double *y)
{
  ShimTest *t = (ShimTest *)h;
  return MFStokesWrapper_A11_B200(&t->mf, &t->volQ, &t->dau, u, y);
}

int shimtest_diag(void *h, double *y)
{
  ShimTest *t = (ShimTest *)h;
  return MFStokesWrapper_diagA11_B200(&t->mf, &t->volQ, &t->dau, y);
}

int shimtest_a12(void *h, double *p, double *yu)
{
  ShimTest *t = (ShimTest *)h;
  return MFStokesWrapper_A12_B200(&t->volQ, &t->dau, NULL, p, yu);
}

int shimtest_a21(void *h, double *u, double *yp)
{
  ShimTest *t = (ShimTest *)h;
  return MFStokesWrapper_A21_B200(&t->volQ, &t->dau, NULL, u, yp);
}

int shimtest_stokes_a(void *h, double *u, double *p, double *yu, double *yp)
{
  ShimTest *t = (ShimTest *)h;
  return MFStokesWrapper_A_B200(&t->stokes, &t->volQ, &t->dau, u, NULL, p, yu, yp);
}

/* The application moved the mesh: new coordinates, new Vec state. */
void shimtest_move(void *h, double *coords)
{
  ShimTest *t = (ShimTest *)h;
  t->dau.coords.a = coords;
  t->dau.coords.hdr.state++;
}

/* New viscosity in the quadrature records; bump_mats: the Mats' states
 * change with it, as after an assembly. */
void shimtest_set_eta(void *h, const double *eta, int bump_mats)
{
  ShimTest *t = (ShimTest *)h;
  PetscInt e;
  for (e = 0; e < 27 * t->nel; e++) t->qp[e].eta = eta[e];
  if (bump_mats) {
    t->mf.state++;
    t->stokes.hdr.state++;
  }
}

void *shimtest_op(void *h)
{
  ShimTest *t = (ShimTest *)h;
  pt_op *op = NULL;
  if (MFA11B200GetOp(&t->dau, &op)) return NULL;
  return op;
}

int shimtest_destroy(void *h)
{
  ShimTest *t = (ShimTest *)h;
  int i, ierr;
  if (!t) return 0;
  ierr = MFA11Destroy_B200(&t->mf);
  for (i = 0; i < MAX_COMPOSED; i++) /* the DM's own reference to the op */
    if (t->dau.hdr.composed[i]) obj_release(t->dau.hdr.composed[i]);
  free(t->qp);
  free(t);
  return ierr;
}
