/*
 * Minimal stand-in for the PETSc 3.8 / MPI declarations that the reference's
 * operator sources and their header closure name.  It only has to make those
 * files compile for one process; the arrays they read are supplied by
 * ref_glue.c.  Used by oracle/Makefile's Route-A target only (test
 * infrastructure).
 */
#ifndef PETSC_STUB_CORE_H
#define PETSC_STUB_CORE_H
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>
#include <math.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef int MPI_Win;
typedef long MPI_Aint;
#define MPI_DOUBLE 1
int MPI_Get_address(const void *, MPI_Aint *);
int MPI_Type_create_struct(int, const int *, const MPI_Aint *, const MPI_Datatype *, MPI_Datatype *);
int MPI_Type_commit(MPI_Datatype *);
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;
#define MPI_COMM_WORLD 0
#define MPI_COMM_SELF 1

typedef int PetscErrorCode;
typedef int PetscInt;
typedef int PetscMPIInt;
typedef int PetscClassId;
typedef int PetscLogEvent;
typedef int PetscLogStage;
typedef double PetscReal;
typedef double PetscScalar;
typedef double PetscLogDouble;
typedef int64_t PetscInt64;
typedef int64_t PetscObjectState;
typedef enum { PETSC_FALSE = 0, PETSC_TRUE = 1 } PetscBool;
typedef enum { INSERT_VALUES, ADD_VALUES } InsertMode;
typedef enum { PETSC_VIEWER_DEFAULT, PETSC_VIEWER_ASCII_VTK } PetscViewerFormat;
typedef enum { DM_BOUNDARY_NONE, DM_BOUNDARY_GHOSTED, DM_BOUNDARY_MIRROR, DM_BOUNDARY_PERIODIC } DMBoundaryType;
typedef enum { DMDA_STENCIL_STAR, DMDA_STENCIL_BOX } DMDAStencilType;
typedef enum { PETSC_COPY_VALUES, PETSC_OWN_POINTER, PETSC_USE_POINTER } PetscCopyMode;
typedef enum { NORM_1, NORM_2, NORM_FROBENIUS, NORM_INFINITY } NormType;
typedef struct { PetscInt i, j, k, c; } MatStencil;
typedef struct { PetscScalar x, y, z; } DMDACoor3d;
typedef struct { PetscScalar x, y; } DMDACoor2d;
typedef const char *MatType;
typedef const char *VecType;
typedef const char *KSPType;
typedef const char *PCType;
typedef int PetscDataType;
typedef int SNESConvergedReason;
typedef int KSPConvergedReason;

typedef struct _p_PetscObject *PetscObject;
typedef struct _p_Vec *Vec;
typedef struct _p_Mat *Mat;
typedef struct _p_DM *DM;
typedef struct _p_IS *IS;
typedef struct _p_KSP *KSP;
typedef struct _p_PC *PC;
typedef struct _p_SNES *SNES;
typedef struct _p_TS *TS;
typedef struct _p_PetscViewer *PetscViewer;
typedef struct _p_PetscRandom *PetscRandom;
typedef struct _p_VecScatter *VecScatter;
typedef struct _p_ISLocalToGlobalMapping *ISLocalToGlobalMapping;
typedef struct _p_PetscFunctionList *PetscFunctionList;
typedef struct _p_PetscContainer *PetscContainer;
typedef struct _p_PetscFE *PetscFE;
typedef struct _p_PetscQuadrature *PetscQuadrature;
typedef struct _p_PetscSection *PetscSection;
typedef struct _p_MatNullSpace *MatNullSpace;
typedef struct _p_PetscSF *PetscSF;
typedef struct _p_MatMFFD *MatMFFD;
typedef const char *MatMFFDType;
#define MATMFFD_WP "wp"
typedef struct {
  PetscInt dim, dof, sw;
  PetscInt mx, my, mz;
  PetscInt xs, ys, zs, xm, ym, zm;
  PetscInt gxs, gys, gzs, gxm, gym, gzm;
} DMDALocalInfo;

#define PETSC_EXTERN extern
#define PETSC_STATIC_INLINE static inline
#define PETSC_COMM_WORLD 0
#define PETSC_COMM_SELF 1
#define PETSC_ERR_SUP 56
#define PETSC_ERR_USER 83
#define PETSC_ERR_ARG_SIZ 60
#define PETSC_ERR_ARG_WRONG 62
#define PETSC_ERR_ARG_CORRUPT 64
#define PETSC_ERR_ARG_NULL 85
#define PETSC_ERR_ARG_OUTOFRANGE 63
#define PETSC_ERR_LIB 76
#define PETSC_ERR_MEM 55
#define PETSC_DECIDE -1
#define PETSC_DEFAULT -2
#define PETSC_NULL 0
#define PETSC_MAX_PATH_LEN 4096
#define PETSC_PI 3.14159265358979323846
#define PetscFunctionBegin
#define PetscFunctionBeginUser
#define PetscFunctionReturn(x) return (x)
#define CHKERRQ(x) do { if (x) return (x); } while (0)
#define CHKERRMPI(x) CHKERRQ(x)
#define SETERRQ(c, n, ...) return (n)
#define SETERRQ1(c, n, ...) return (n)
#define SETERRQ2(c, n, ...) return (n)
#define SETERRQ3(c, n, ...) return (n)
#define PetscMin(a, b) (((a) < (b)) ? (a) : (b))
#define PetscMax(a, b) (((a) < (b)) ? (b) : (a))
#define PetscSqr(a) ((a) * (a))
#define PetscSqrtReal(a) sqrt(a)
#define PetscAbsReal(a) fabs(a)
#define PetscPowReal(a, b) pow(a, b)
#define PetscMemzero(a, n) (memset((a), 0, (n)), 0)
#define PetscMemcpy(a, b, n) (memcpy((a), (b), (n)), 0)
#define PetscLogFlops(n) 0
#define PetscMalloc(n, p) ((*(void **)(p) = malloc(n)) == NULL)
#define PetscMalloc1(n, p) ((*(void **)(p) = malloc(sizeof(**(p)) * (n))) == NULL)
#define PetscCalloc1(n, p) ((*(void **)(p) = calloc((n), sizeof(**(p)))) == NULL)
#define PetscFree(p) (free(p), (p) = NULL, 0)
#define PetscPrintf(c, ...) printf(__VA_ARGS__)

/* The routines the operator files call; implemented in ref_glue.c. */
PetscErrorCode PetscDTGaussQuadrature(PetscInt, PetscReal, PetscReal, PetscReal *, PetscReal *);
PetscErrorCode DMGetCoordinateDM(DM, DM *);
PetscErrorCode DMGetCoordinatesLocal(DM, Vec *);
PetscErrorCode VecGetArrayRead(Vec, const PetscScalar **);
PetscErrorCode VecRestoreArrayRead(Vec, const PetscScalar **);
PetscErrorCode VecGetArray(Vec, PetscScalar **);
PetscErrorCode VecRestoreArray(Vec, PetscScalar **);
PetscErrorCode PetscTime(PetscLogDouble *);

/* Declarations for code written against PETSc (the b200 plug-in shim); the
 * shim's test build implements them in shim_host.c, the Route-A build does
 * not use them. */
PetscErrorCode DMDAGetGhostCorners(DM, PetscInt *, PetscInt *, PetscInt *, PetscInt *, PetscInt *, PetscInt *);
PetscErrorCode PetscObjectQuery(PetscObject, const char[], PetscObject *);
PetscErrorCode PetscObjectCompose(PetscObject, const char[], PetscObject);
PetscErrorCode PetscObjectStateGet(PetscObject, PetscObjectState *);
PetscErrorCode PetscObjectReference(PetscObject);
MPI_Comm PetscObjectComm(PetscObject);
PetscErrorCode PetscContainerCreate(MPI_Comm, PetscContainer *);
PetscErrorCode PetscContainerSetPointer(PetscContainer, void *);
PetscErrorCode PetscContainerGetPointer(PetscContainer, void **);
PetscErrorCode PetscContainerSetUserDestroy(PetscContainer, PetscErrorCode (*)(void *));
PetscErrorCode PetscContainerDestroy(PetscContainer *);
PetscErrorCode PetscFunctionListAdd_Private(PetscFunctionList *, const char[], void (*)(void));
#define PetscFunctionListAdd(list, name, fptr) PetscFunctionListAdd_Private((list), (name), (void (*)(void))(fptr))
#endif
