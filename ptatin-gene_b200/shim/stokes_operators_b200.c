/*
 * pTatin3D plug-in for the B200 operator library (libpt_b200.so).
 *
 * Registers the A11 back-end "b200" with the same SpMVOp triple the reference
 * dispatches through (include/stokes_operators.h:61-63):
 *   MFStokesWrapper_A11_B200   -> MatA11MF->SpMVOp_MatMult
 *   MFA11SetUp_B200            -> MatA11MF->SpMVOp_SetUp
 *   MFA11Destroy_B200          -> MatA11MF->SpMVOp_Destroy
 * and provides drop-ins for the hard-wired diag / A12 / A21 element loops
 * (src/stokes_operators.c:1094, 1339-1343, 1479):
 *   MFStokesWrapper_diagA11_B200, MFStokesWrapper_A12_B200, MFStokesWrapper_A21_B200,
 * and for the whole Stokes operator of MatMult_MFStokes_A (stokes_operators.c:937-941):
 *   MFStokesWrapper_A_B200.
 *
 * Contract, identical to the CPU back-ends (src/stokes_operators_tensor.c:181):
 * ufield/Xp/Xu are the rank's ghosted local arrays (Dirichlet entries already
 * zeroed by the caller), the output array is the zeroed local vector that the
 * caller scatters with DMLocalToGlobal(ADD_VALUES) and then fixes the BC rows.
 * The back-end does no BC work.  Errors come back as PetscErrorCode; the
 * library never exits the process.
 *
 * Device data.  One pt_op per velocity DM holds the coordinates, the
 * quadrature-point viscosity and everything derived from them (the Gauss-point
 * geometry factors, the divergence blocks); the A11 shell (mf->ctx) and the
 * diag / B / B^T / whole-operator calls all use it, so a run keeps one copy.
 *   - coordinates are uploaded when the coordinate Vec (or its
 *     PetscObjectState) changes, i.e. when the mesh moves;
 *   - the viscosity is uploaded when the state of the calling Mat changes, as
 *     the reference CUDA back-end does with mf->state
 *     (src/stokes_operators_cuda.cu:413-422).  Each calling Mat (the A11 shell
 *     for MatMult and MatGetDiagonal, the Stokes shell for the whole operator)
 *     is tracked by its own last-seen state.
 * Only an upload invalidates the derived data, so repeated MatMults with
 * unchanged coordinates and viscosity run the kernels alone.
 *
 * Build (where PETSc and pTatin3D are available): compile this file with the
 * pTatin3D include path and -I<repo>/include, link -lpt_b200.
 */
#include <petsc.h>
#include <petscdm.h>

#include "ptatin3d.h"
#include "private/ptatin_impl.h"
#include "ptatin3d_stokes.h"
#include "dmda_element_q2p1.h"
#include "stokes_operators.h"

#include "pt_b200.h"

#define B200_ETA_KEYS 8

/* The op shared by every caller on one velocity DM. */
typedef struct {
  pt_op *op;
  Vec coords_vec;                 /* the coordinate Vec last uploaded ... */
  PetscObjectState coords_state;  /* ... and its state then */
  PetscBool have_coords, have_eta;
  struct {
    const void *key;              /* the calling Mat */
    PetscObjectState state;       /* its state at the last viscosity upload it saw */
  } eta_seen[B200_ETA_KEYS];
  int n_seen, next_slot;
} B200Op;

/* mf->ctx of the A11 shell: a reference to the DM's op. */
typedef struct {
  PetscContainer cont;
  B200Op *b;
} MFA11B200;

#define PTCHK(call)                                                                                 \
  do {                                                                                              \
    pt_status _s = (call);                                                                          \
    if (_s != PT_OK) SETERRQ2(PETSC_COMM_SELF, PETSC_ERR_LIB, "%s: %s", #call, pt_last_error());     \
  } while (0)

/* Local element box of this rank in its ghosted node box, as the element table
 * of dmda_element_q2p1.c:395-455 numbers it (node (esi-gsi)+2ei+c, ...). */
static PetscErrorCode B200_MeshDesc(DM dau, pt_mesh_desc *d)
{
  PetscErrorCode ierr;
  PetscInt sei, sej, sek, mx, my, mz, gsi, gsj, gsk, X, Y, Z;

  PetscFunctionBegin;
  ierr = DMDAGetCornersElementQ2(dau, &sei, &sej, &sek, &mx, &my, &mz);CHKERRQ(ierr);
  ierr = DMDAGetGhostCorners(dau, &gsi, &gsj, &gsk, &X, &Y, &Z);CHKERRQ(ierr);
  memset(d, 0, sizeof *d);
  d->mx = (int32_t)mx; d->my = (int32_t)my; d->mz = (int32_t)mz;
  d->nx = (int32_t)X;  d->ny = (int32_t)Y;  d->nz = (int32_t)Z;
  d->ox = (int32_t)(sei - gsi); d->oy = (int32_t)(sej - gsj); d->oz = (int32_t)(sek - gsk);
  PetscFunctionReturn(0);
}

static PetscErrorCode B200_OpDestroy(void *ctx)
{
  B200Op *b = (B200Op *)ctx;
  if (b) {
    pt_op_destroy(b->op);
    PetscFree(b);
  }
  return 0;
}

/* The op composed on dau ("pt_b200_op"), created on first use; the DM holds
 * the only reference unless *cont_ref is asked for (then the caller owns one
 * more and releases it with PetscContainerDestroy). */
static PetscErrorCode B200_Shared(DM dau, B200Op **out, PetscContainer *cont_ref)
{
  PetscErrorCode ierr;
  PetscContainer cont = NULL;
  B200Op *b;

  PetscFunctionBegin;
  ierr = PetscObjectQuery((PetscObject)dau, "pt_b200_op", (PetscObject *)&cont);CHKERRQ(ierr);
  if (!cont) {
    pt_mesh_desc d;
    ierr = B200_MeshDesc(dau, &d);CHKERRQ(ierr);
    ierr = PetscCalloc1(1, &b);CHKERRQ(ierr);
    if (pt_op_create(&d, &b->op) != PT_OK) {
      ierr = PetscFree(b);CHKERRQ(ierr);
      SETERRQ1(PETSC_COMM_SELF, PETSC_ERR_LIB, "pt_op_create: %s", pt_last_error());
    }
    ierr = PetscContainerCreate(PetscObjectComm((PetscObject)dau), &cont);CHKERRQ(ierr);
    ierr = PetscContainerSetPointer(cont, b);CHKERRQ(ierr);
    ierr = PetscContainerSetUserDestroy(cont, B200_OpDestroy);CHKERRQ(ierr);
    ierr = PetscObjectCompose((PetscObject)dau, "pt_b200_op", (PetscObject)cont);CHKERRQ(ierr);
    ierr = PetscContainerDestroy(&cont);CHKERRQ(ierr);
    ierr = PetscObjectQuery((PetscObject)dau, "pt_b200_op", (PetscObject *)&cont);CHKERRQ(ierr);
  }
  ierr = PetscContainerGetPointer(cont, (void **)&b);CHKERRQ(ierr);
  if (cont_ref) {
    ierr = PetscObjectReference((PetscObject)cont);CHKERRQ(ierr);
    *cont_ref = cont;
  }
  *out = b;
  PetscFunctionReturn(0);
}

/* Brings the op's coordinates (and, with need_eta, viscosity) up to date:
 * coordinates when the coordinate Vec or its state changed, viscosity when the
 * calling Mat `key` shows a state other than the one it showed at its last
 * upload (or has never been seen).  QPntVolCoefStokes is a 48-byte record
 * with eta at offset 0 (include/QPntVolCoefStokes_def.h:41-46). */
static PetscErrorCode B200_Sync(B200Op *b, DM dau, Quadrature volQ, const void *key, PetscObjectState key_state,
                                PetscBool need_eta)
{
  PetscErrorCode ierr;
  Vec gcoords;
  PetscObjectState st;

  PetscFunctionBegin;
  ierr = DMGetCoordinatesLocal(dau, &gcoords);CHKERRQ(ierr);
  ierr = PetscObjectStateGet((PetscObject)gcoords, &st);CHKERRQ(ierr);
  if (!b->have_coords || b->coords_vec != gcoords || b->coords_state != st) {
    const PetscScalar *LA_gcoords;
    ierr = VecGetArrayRead(gcoords, &LA_gcoords);CHKERRQ(ierr);
    PTCHK(pt_op_set_coords_h(b->op, LA_gcoords));
    ierr = VecRestoreArrayRead(gcoords, &LA_gcoords);CHKERRQ(ierr);
    b->coords_vec = gcoords;
    b->coords_state = st;
    b->have_coords = PETSC_TRUE;
  }
  if (need_eta) {
    int i, hit = -1;
    for (i = 0; i < b->n_seen; i++)
      if (b->eta_seen[i].key == key) hit = i;
    if (!b->have_eta || hit < 0 || b->eta_seen[hit].state != key_state) {
      QPntVolCoefStokes *qp;
      ierr = VolumeQuadratureGetAllCellData_Stokes(volQ, &qp);CHKERRQ(ierr);
      PTCHK(pt_op_set_eta_strided_h(b->op, &qp[0].eta, (int64_t)(sizeof(QPntVolCoefStokes) / sizeof(double))));
      b->have_eta = PETSC_TRUE;
      if (hit < 0) {
        hit = b->n_seen < B200_ETA_KEYS ? b->n_seen++ : (b->next_slot++ % B200_ETA_KEYS);
        b->eta_seen[hit].key = key;
      }
      b->eta_seen[hit].state = key_state;
    }
  }
  PetscFunctionReturn(0);
}

/* The op of the velocity DM, for callers that want to hand it to the device
 * solver (pt_solver_create) or read its counters. */
PetscErrorCode MFA11B200GetOp(DM dau, pt_op **op)
{
  PetscErrorCode ierr;
  B200Op *b;

  PetscFunctionBeginUser;
  ierr = B200_Shared(dau, &b, NULL);CHKERRQ(ierr);
  *op = b->op;
  PetscFunctionReturn(0);
}

/* ---- SpMVOp triple -------------------------------------------------------- */

PetscErrorCode MFA11SetUp_B200(MatA11MF mf)
{
  PetscErrorCode ierr;
  MFA11B200 *c;

  PetscFunctionBeginUser;
  if (mf->ctx) PetscFunctionReturn(0);
  ierr = PetscCalloc1(1, &c);CHKERRQ(ierr);
  ierr = B200_Shared(mf->daUVW, &c->b, &c->cont);CHKERRQ(ierr);
  mf->ctx = c;
  PetscFunctionReturn(0);
}

PetscErrorCode MFStokesWrapper_A11_B200(MatA11MF mf, Quadrature volQ, DM dau, PetscScalar ufield[], PetscScalar Yu[])
{
  PetscErrorCode ierr;
  MFA11B200 *c = (MFA11B200 *)mf->ctx;

  PetscFunctionBeginUser;
  if (!c) SETERRQ(PETSC_COMM_SELF, PETSC_ERR_USER, "b200 MF-SpMV implementation should have a valid context");
  ierr = B200_Sync(c->b, dau, volQ, mf, mf->state, PETSC_TRUE);CHKERRQ(ierr);
  /* Yu was zeroed by the caller (stokes_operators.c:1195-1196): overwrite == add */
  PTCHK(pt_a11_apply_h(c->b->op, ufield, Yu));
  PetscFunctionReturn(0);
}

PetscErrorCode MFA11Destroy_B200(MatA11MF mf)
{
  PetscErrorCode ierr;
  MFA11B200 *c = (MFA11B200 *)mf->ctx;

  PetscFunctionBeginUser;
  if (!c) SETERRQ(PETSC_COMM_SELF, PETSC_ERR_USER, "b200 MF-SpMV implementation should have a valid context");
  ierr = PetscContainerDestroy(&c->cont);CHKERRQ(ierr);
  ierr = PetscFree(c);CHKERRQ(ierr);
  mf->ctx = NULL;
  PetscFunctionReturn(0);
}

/* Adds "b200" to the three function lists of MatA11MFCreate
 * (src/stokes_operators.c:123-142). */
PetscErrorCode MatA11MFRegister_B200(PetscFunctionList *matmult, PetscFunctionList *setup, PetscFunctionList *destroy)
{
  PetscErrorCode ierr;

  PetscFunctionBeginUser;
  ierr = PetscFunctionListAdd(matmult, "b200", MFStokesWrapper_A11_B200);CHKERRQ(ierr);
  ierr = PetscFunctionListAdd(setup, "b200", MFA11SetUp_B200);CHKERRQ(ierr);
  ierr = PetscFunctionListAdd(destroy, "b200", MFA11Destroy_B200);CHKERRQ(ierr);
  PetscFunctionReturn(0);
}

/* ---- diag / B / B^T / the whole operator ------------------------------------ */

/* Replaces MFStokesWrapper_diagA11 (src/stokes_operators_mf.c:71-135) inside
 * MatGetDiagonal_MFStokes_A11, which passes its MatA11MF with mf->state set
 * from the Mat (as MatMult_MFStokes_A11 does, stokes_operators.c:1176-1177). */
PetscErrorCode MFStokesWrapper_diagA11_B200(MatA11MF mf, Quadrature volQ, DM dau, PetscScalar Yu[])
{
  PetscErrorCode ierr;
  B200Op *b;

  PetscFunctionBeginUser;
  if (mf->ctx) b = ((MFA11B200 *)mf->ctx)->b;
  else {
    ierr = B200_Shared(dau, &b, NULL);CHKERRQ(ierr);
  }
  ierr = B200_Sync(b, dau, volQ, mf, mf->state, PETSC_TRUE);CHKERRQ(ierr);
  PTCHK(pt_a11_diag_h(b->op, Yu));
  PetscFunctionReturn(0);
}

/* Replaces MFStokesWrapper_A12_AVX / MFStokesWrapper_A12 (stokes_operators_avx.c:682,
 * stokes_operators_mf.c:792).  Pressure is element-local (4 dofs per element);
 * B^T depends on the coordinates only. */
PetscErrorCode MFStokesWrapper_A12_B200(Quadrature volQ, DM dau, DM dap, PetscScalar Xp[], PetscScalar Yu[])
{
  PetscErrorCode ierr;
  B200Op *b;

  PetscFunctionBeginUser;
  (void)dap;
  ierr = B200_Shared(dau, &b, NULL);CHKERRQ(ierr);
  ierr = B200_Sync(b, dau, volQ, NULL, 0, PETSC_FALSE);CHKERRQ(ierr);
  PTCHK(pt_a12_apply_h(b->op, Xp, Yu));
  PetscFunctionReturn(0);
}

/* Replaces MFStokesWrapper_A21 (src/stokes_operators_mf.c:862-937). */
PetscErrorCode MFStokesWrapper_A21_B200(Quadrature volQ, DM dau, DM dap, PetscScalar Xu[], PetscScalar Yp[])
{
  PetscErrorCode ierr;
  B200Op *b;

  PetscFunctionBeginUser;
  (void)dap;
  ierr = B200_Shared(dau, &b, NULL);CHKERRQ(ierr);
  ierr = B200_Sync(b, dau, volQ, NULL, 0, PETSC_FALSE);CHKERRQ(ierr);
  PTCHK(pt_a21_apply_h(b->op, Xu, Yp));
  PetscFunctionReturn(0);
}

/* Replaces MFStokesWrapper_A_AVX / MFStokesWrapper_A (stokes_operators_avx.c:439,
 * stokes_operators_mf.c:711) inside MatMult_MFStokes_A: Yu = A11 u + A12 p,
 * Yp = A21 u in one call.  A is the Stokes shell whose state versions the
 * viscosity. */
PetscErrorCode MFStokesWrapper_A_B200(Mat A, Quadrature volQ, DM dau, PetscScalar ufield[], DM dap,
                                      PetscScalar pfield[], PetscScalar Yu[], PetscScalar Yp[])
{
  PetscErrorCode ierr;
  B200Op *b;
  PetscObjectState st;

  PetscFunctionBeginUser;
  (void)dap;
  ierr = PetscObjectStateGet((PetscObject)A, &st);CHKERRQ(ierr);
  ierr = B200_Shared(dau, &b, NULL);CHKERRQ(ierr);
  ierr = B200_Sync(b, dau, volQ, A, st, PETSC_TRUE);CHKERRQ(ierr);
  PTCHK(pt_stokes_a_apply_h(b->op, ufield, pfield, Yu, Yp));
  PetscFunctionReturn(0);
}
