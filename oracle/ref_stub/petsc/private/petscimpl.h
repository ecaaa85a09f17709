/* PETSc stand-in (test infrastructure): what the reference's vendored copy of
 * PETSc 3.13's mffdimpl.h (include/petsc/src/mat/impls/mffd/mffdimpl.h) needs
 * to declare its context struct. */
#include "petsc_stub_core.h"
typedef struct _p_PetscOptionItems PetscOptionItems;
#define PETSCHEADER(ObjectOps) \
  struct {                     \
    int classid;               \
  } hdr;                       \
  ObjectOps *ops
