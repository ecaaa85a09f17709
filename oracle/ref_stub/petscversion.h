/* PETSc stand-in (test infrastructure): the version the reference's private
 * MFFD header checks for (include/petsc/ptatin_petsc_mffdimpl.h). */
#include "petsc_stub_core.h"
#define PETSC_VERSION_MAJOR 3
#define PETSC_VERSION_MINOR 13
#define PETSC_VERSION_SUBMINOR 0
