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
 * The back-end does no BC work.  Coordinates and quadrature-point viscosity
 * are uploaded when the Mat's PetscObjectState changes (mf->state), as the
 * reference CUDA back-end does (src/stokes_operators_cuda.cu:413-422), and
 * otherwise stay resident in HBM.  Errors come back as PetscErrorCode; the
 * library never exits the process.
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

typedef struct {
  pt_op *op;
  PetscObjectState state; /* state of the uploaded coordinates / viscosity */
  PetscBool have_data;
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

static PetscErrorCode B200_Create(DM dau, MFA11B200 **out)
{
  PetscErrorCode ierr;
  pt_mesh_desc d;
  MFA11B200 *c;

  PetscFunctionBegin;
  ierr = B200_MeshDesc(dau, &d);CHKERRQ(ierr);
  ierr = PetscCalloc1(1, &c);CHKERRQ(ierr);
  PTCHK(pt_op_create(&d, &c->op));
  c->state = -1;
  *out = c;
  PetscFunctionReturn(0);
}

/* Upload coordinates and eta (QPntVolCoefStokes AoS, eta at offset 0). */
static PetscErrorCode B200_Upload(MFA11B200 *c, Quadrature volQ, DM dau, PetscBool need_eta)
{
  PetscErrorCode ierr;
  Vec gcoords;
  const PetscScalar *LA_gcoords;
  QPntVolCoefStokes *qp;

  PetscFunctionBegin;
  ierr = DMGetCoordinatesLocal(dau, &gcoords);CHKERRQ(ierr);
  ierr = VecGetArrayRead(gcoords, &LA_gcoords);CHKERRQ(ierr);
  PTCHK(pt_op_set_coords_h(c->op, LA_gcoords));
  ierr = VecRestoreArrayRead(gcoords, &LA_gcoords);CHKERRQ(ierr);
  if (need_eta) {
    ierr = VolumeQuadratureGetAllCellData_Stokes(volQ, &qp);CHKERRQ(ierr);
    PTCHK(pt_op_set_eta_strided_h(c->op, &qp[0].eta, (int64_t)(sizeof(QPntVolCoefStokes) / sizeof(double))));
  }
  c->have_data = PETSC_TRUE;
  PetscFunctionReturn(0);
}

/* ---- SpMVOp triple -------------------------------------------------------- */

PetscErrorCode MFA11SetUp_B200(MatA11MF mf)
{
  PetscErrorCode ierr;
  MFA11B200 *c;

  PetscFunctionBeginUser;
  if (mf->ctx) PetscFunctionReturn(0);
  ierr = B200_Create(mf->daUVW, &c);CHKERRQ(ierr);
  mf->ctx = c;
  PetscFunctionReturn(0);
}

PetscErrorCode MFStokesWrapper_A11_B200(MatA11MF mf, Quadrature volQ, DM dau, PetscScalar ufield[], PetscScalar Yu[])
{
  PetscErrorCode ierr;
  MFA11B200 *c = (MFA11B200 *)mf->ctx;

  PetscFunctionBeginUser;
  if (!c) SETERRQ(PETSC_COMM_SELF, PETSC_ERR_USER, "b200 MF-SpMV implementation should have a valid context");
  if (!c->have_data || c->state != mf->state) {
    ierr = B200_Upload(c, volQ, dau, PETSC_TRUE);CHKERRQ(ierr);
    c->state = mf->state;
  }
  /* Yu was zeroed by the caller (stokes_operators.c:1195-1196): overwrite == add */
  PTCHK(pt_a11_apply_h(c->op, ufield, Yu));
  PetscFunctionReturn(0);
}

PetscErrorCode MFA11Destroy_B200(MatA11MF mf)
{
  PetscErrorCode ierr;
  MFA11B200 *c = (MFA11B200 *)mf->ctx;

  PetscFunctionBeginUser;
  if (!c) SETERRQ(PETSC_COMM_SELF, PETSC_ERR_USER, "b200 MF-SpMV implementation should have a valid context");
  PTCHK(pt_op_destroy(c->op));
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

/* ---- diag / B / B^T: one op cached on the velocity DM ---------------------- */

static PetscErrorCode B200_ContainerDestroy(void *ctx)
{
  MFA11B200 *c = (MFA11B200 *)ctx;
  if (c) {
    pt_op_destroy(c->op);
    PetscFree(c);
  }
  return 0;
}

static PetscErrorCode B200_GetCached(DM dau, Quadrature volQ, PetscBool need_eta, MFA11B200 **out)
{
  PetscErrorCode ierr;
  PetscContainer cont = NULL;
  MFA11B200 *c;
  PetscObjectState st;

  PetscFunctionBegin;
  ierr = PetscObjectQuery((PetscObject)dau, "pt_b200_op", (PetscObject *)&cont);CHKERRQ(ierr);
  if (!cont) {
    ierr = B200_Create(dau, &c);CHKERRQ(ierr);
    ierr = PetscContainerCreate(PetscObjectComm((PetscObject)dau), &cont);CHKERRQ(ierr);
    ierr = PetscContainerSetPointer(cont, c);CHKERRQ(ierr);
    ierr = PetscContainerSetUserDestroy(cont, B200_ContainerDestroy);CHKERRQ(ierr);
    ierr = PetscObjectCompose((PetscObject)dau, "pt_b200_op", (PetscObject)cont);CHKERRQ(ierr);
    ierr = PetscContainerDestroy(&cont);CHKERRQ(ierr);
  } else {
    ierr = PetscContainerGetPointer(cont, (void **)&c);CHKERRQ(ierr);
  }
  /* the coordinate Vec's state tracks mesh motion; re-upload when it moves */
  {
    Vec gcoords;
    ierr = DMGetCoordinatesLocal(dau, &gcoords);CHKERRQ(ierr);
    ierr = PetscObjectStateGet((PetscObject)gcoords, &st);CHKERRQ(ierr);
  }
  if (!c->have_data || c->state != st || need_eta) {
    ierr = B200_Upload(c, volQ, dau, need_eta);CHKERRQ(ierr);
    c->state = st;
  }
  *out = c;
  PetscFunctionReturn(0);
}

/* Replaces MFStokesWrapper_diagA11 (src/stokes_operators_mf.c:71-135). */
PetscErrorCode MFStokesWrapper_diagA11_B200(Quadrature volQ, DM dau, PetscScalar Yu[])
{
  PetscErrorCode ierr;
  MFA11B200 *c;

  PetscFunctionBeginUser;
  ierr = B200_GetCached(dau, volQ, PETSC_TRUE, &c);CHKERRQ(ierr);
  PTCHK(pt_a11_diag_h(c->op, Yu));
  PetscFunctionReturn(0);
}

/* Replaces MFStokesWrapper_A12_AVX / MFStokesWrapper_A12 (stokes_operators_avx.c:682,
 * stokes_operators_mf.c:792).  Pressure is element-local (4 dofs per element). */
PetscErrorCode MFStokesWrapper_A12_B200(Quadrature volQ, DM dau, DM dap, PetscScalar Xp[], PetscScalar Yu[])
{
  PetscErrorCode ierr;
  MFA11B200 *c;

  PetscFunctionBeginUser;
  (void)dap;
  ierr = B200_GetCached(dau, volQ, PETSC_FALSE, &c);CHKERRQ(ierr);
  PTCHK(pt_a12_apply_h(c->op, Xp, Yu));
  PetscFunctionReturn(0);
}

/* Replaces MFStokesWrapper_A_AVX / MFStokesWrapper_A (stokes_operators_avx.c:439,
 * stokes_operators_mf.c:711): Yu = A11 u + A12 p, Yp = A21 u in one call. */
PetscErrorCode MFStokesWrapper_A_B200(Quadrature volQ, DM dau, PetscScalar ufield[], DM dap, PetscScalar pfield[],
                                      PetscScalar Yu[], PetscScalar Yp[])
{
  PetscErrorCode ierr;
  MFA11B200 *c;

  PetscFunctionBeginUser;
  (void)dap;
  ierr = B200_GetCached(dau, volQ, PETSC_TRUE, &c);CHKERRQ(ierr);
  PTCHK(pt_stokes_a_apply_h(c->op, ufield, pfield, Yu, Yp));
  PetscFunctionReturn(0);
}

/* Replaces MFStokesWrapper_A21 (src/stokes_operators_mf.c:862-937). */
PetscErrorCode MFStokesWrapper_A21_B200(Quadrature volQ, DM dau, DM dap, PetscScalar Xu[], PetscScalar Yp[])
{
  PetscErrorCode ierr;
  MFA11B200 *c;

  PetscFunctionBeginUser;
  (void)dap;
  ierr = B200_GetCached(dau, volQ, PETSC_FALSE, &c);CHKERRQ(ierr);
  PTCHK(pt_a21_apply_h(c->op, Xu, Yp));
  PetscFunctionReturn(0);
}
