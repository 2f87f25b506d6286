/* TEST INFRASTRUCTURE ONLY: the PETSc subset the B200Rhs process (ablate_b200/reference_process) uses,
 * so that it compiles and runs here without PETSc: scalar types, error codes and macros, and a Vec that
 * is a plain host array. The real PETSc headers replace this file in an ABLATE build. */
#pragma once
#include <cstdarg>
#include <cstdio>
#include <string>

typedef double PetscReal;
typedef double PetscScalar;
typedef int PetscInt;
typedef int PetscErrorCode;
#define PETSC_SUCCESS 0
#define PETSC_ERR_LIB 76
#define PETSC_ERR_ARG_WRONGSTATE 73
#define PETSC_COMM_SELF 0

struct _p_Vec {
    PetscScalar* array = nullptr;
    PetscInt n = 0;
};
typedef _p_Vec* Vec;
struct _p_DM {};
typedef _p_DM* DM;

namespace petsc_shim {
// the text of the last error raised with SETERRQ
inline std::string& last_error() {
    static std::string s;
    return s;
}
inline PetscErrorCode raise(PetscErrorCode code, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    last_error() = buf;
    return code;
}
}  // namespace petsc_shim

#define PetscFunctionBeginUser
#define PetscFunctionReturn(x) return (x)
#define PetscCall(x)                          \
    do {                                      \
        PetscErrorCode e_ = (x);              \
        if (e_ != PETSC_SUCCESS) return e_;   \
    } while (0)
#define SETERRQ(comm, code, ...) return petsc_shim::raise(code, __VA_ARGS__)

inline PetscErrorCode VecGetArrayRead(Vec v, const PetscScalar** a) {
    *a = v->array;
    return PETSC_SUCCESS;
}
inline PetscErrorCode VecRestoreArrayRead(Vec, const PetscScalar** a) {
    *a = nullptr;
    return PETSC_SUCCESS;
}
inline PetscErrorCode VecGetArray(Vec v, PetscScalar** a) {
    *a = v->array;
    return PETSC_SUCCESS;
}
inline PetscErrorCode VecRestoreArray(Vec, PetscScalar** a) {
    *a = nullptr;
    return PETSC_SUCCESS;
}
