/*
 * Route-A glue: placeholder definitions for PETSc / pTatin3D routines that the
 * reference's src/material_point_utils.c and the struct-definition sources
 * reference outside the marker -> Gauss-point projection path (viewers, MPI
 * data types, multigrid hierarchies, surface quadrature, data buckets).  They
 * let libptref.so load; none is called by the entry points of ref_glue.c, and
 * each returns an error code if it ever were.  TEST INFRASTRUCTURE ONLY.
 */
int DMCreateInjection(void) { return 73; }
int DMCreateInterpolationScale(void) { return 73; }
int DMDADuplicateLayout(void) { return 73; }
int DMDAEQ1_GetElementLocalIndicesDOF(void) { return 73; }
int DMDAEQ1_GetScalarElementField_3D(void) { return 73; }
int DMDAEQ1_SetValuesLocalStencil_AddValues_DOF(void) { return 73; }
int DMDAGetElementsQ1(void) { return 73; }
int DMDAGetLocalSizeElementQ2(void) { return 73; }
int DMDAGetRefinementFactor(void) { return 73; }
int DMDASetElementType_Q2(void) { return 73; }
int DMDestroy(void) { return 73; }
int DMGetGlobalVector(void) { return 73; }
int DMRestoreGlobalVector(void) { return 73; }
int DMView(void) { return 73; }
int MPI_Comm_rank(void) { return 73; }
int MPI_Comm_size(void) { return 73; }
int MPI_Get_address(void) { return 73; }
int MPI_Type_commit(void) { return 73; }
int MPI_Type_create_struct(void) { return 73; }
int MatDestroy(void) { return 73; }
int MatMult(void) { return 73; }
int MatRestrict(void) { return 73; }
int PetscMPIIntCast(void) { return 73; }
int PetscObjectSetName(void) { return 73; }
int PetscOptionsGetBool(void) { return 73; }
int PetscOptionsGetInt(void) { return 73; }
int PetscSNPrintf(void) { return 73; }
int PetscViewerASCIIOpen(void) { return 73; }
int PetscViewerDestroy(void) { return 73; }
int PetscViewerPopFormat(void) { return 73; }
int PetscViewerPushFormat(void) { return 73; }
int SurfaceQuadratureGetAllCellData_Stokes(void) { return 73; }
int SurfaceQuadratureGetCellData_Stokes(void) { return 73; }
int SurfaceQuadratureViewParaview_Stokes2(void) { return 73; }
int VecDestroy(void) { return 73; }
int VecPointwiseMult(void) { return 73; }
int VecReciprocal(void) { return 73; }
int VecView(void) { return 73; }
int pTatinGenerateParallelVTKName(void) { return 73; }
int pTatinGenerateVTKName(void) { return 73; }
int ptatinDataBucketGetDataFieldByName(void) { return 73; }
int ptatinDataBucketGetDataFields(void) { return 73; }
int ptatinDataBucketGetSizes(void) { return 73; }
int ptatinDataBucketQueryDataFieldByName(void) { return 73; }
int ptatinDataFieldAccessPoint(void) { return 73; }
int ptatinDataFieldGetAccess(void) { return 73; }
int ptatinDataFieldRestoreAccess(void) { return 73; }
int ptatinDataFieldVerifyAccess(void) { return 73; }

/* Referenced by src/stokes_form_function.c outside FormFunctionLocal_U (the
 * SNES residual / matrix-free Jacobian drivers and their PETSc plumbing). */
int BCListInsertDirichlet_MatMult(void) { return 73; }
int BCListInsertLocal(void) { return 73; }
int BCListInsertLocalZero(void) { return 73; }
int BCListResidualDirichlet(void) { return 73; }
int DMCompositeGather(void) { return 73; }
int DMCompositeGetAccess(void) { return 73; }
int DMCompositeGetEntries(void) { return 73; }
int DMCompositeGetLocalVectors(void) { return 73; }
int DMCompositeRestoreAccess(void) { return 73; }
int DMCompositeRestoreLocalVectors(void) { return 73; }
int DMCompositeScatter(void) { return 73; }
int DMCreateGlobalVector(void) { return 73; }
int DMCreateLocalVector(void) { return 73; }
int DMDAGetLocalInfo(void) { return 73; }
int DMGetCoordinates(void) { return 73; }
int MatCreateMFFD(void) { return 73; }
int MatCreateVecs(void) { return 73; }
int MatMFFDResetHHistory(void) { return 73; }
int MatMFFDSetFunction(void) { return 73; }
int MatMFFDSetType(void) { return 73; }
int PetscObjectGetComm(void) { return 73; }
int SurfaceConstraintOps_EvaluateFp(void) { return 73; }
int SurfaceConstraintOps_EvaluateFu(void) { return 73; }
int VecAXPY(void) { return 73; }
int VecCopy(void) { return 73; }
int VecDuplicate(void) { return 73; }
int VecGetLocalSize(void) { return 73; }
int VecGetSize(void) { return 73; }
int pTatinGetStokesContext(void) { return 73; }
int pTatinModel_ApplyBoundaryCondition(void) { return 73; }
int pTatin_EvaluateRheologyNonlinearities(void) { return 73; }
