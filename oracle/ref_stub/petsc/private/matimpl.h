/* PETSc stand-in (test infrastructure): the members of PETSc's private Mat
 * that src/stokes_form_function.c touches (Jij->data, the MFFD context;
 * J->assembled).  Those routines are compiled but never called. */
#include "petsc_stub_core.h"
struct _p_Mat {
  void *data;
  PetscBool assembled;
};
