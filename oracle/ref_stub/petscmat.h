#include "petsc_stub_core.h"
