/* TEST INFRASTRUCTURE ONLY: the few PETSc scalar types and math macros the reference's flux-calculator
 * sources use, so that those files compile here unchanged (PETSc itself is not available). */
#pragma once
#include <cmath>
#include <memory>
#include <stdexcept>
#include <string>
typedef double PetscReal;
typedef double PetscScalar;
typedef int PetscInt;
#define PetscSqr(a) ((a) * (a))
#define PetscAbsReal(a) (std::fabs(a))
#define PetscAbs(a) (std::fabs(a))
#define PetscSqrtReal(a) (std::sqrt(a))
#define PetscPowReal(a, b) (std::pow(a, b))
#define PetscMin(a, b) (((a) < (b)) ? (a) : (b))
#define PetscMax(a, b) (((a) < (b)) ? (b) : (a))
