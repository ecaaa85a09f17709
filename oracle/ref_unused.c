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
