/* Type-only stand-in for the PETSc headers the frehg2 sources include.
 * Test infrastructure: the reference's LinearSystem.cpp is replaced by
 * oracle/shim/linear_system_shim.cpp, which restates PETSc KSPCG semantics,
 * so only the handle and scalar types are needed here. */
#ifndef FREHG_SHIM_PETSCKSP_H
#define FREHG_SHIM_PETSCKSP_H

#include <stdint.h>

typedef int PetscInt;
typedef int64_t PetscCount;
typedef double PetscReal;
typedef double PetscScalar;
typedef int PetscErrorCode;
typedef enum { PETSC_FALSE = 0, PETSC_TRUE = 1 } PetscBool;
typedef struct _p_Mat* Mat;
typedef struct _p_Vec* Vec;
typedef struct _p_KSP* KSP;
typedef struct _p_PC* PC;
typedef const char* MatType;
typedef const char* VecType;

typedef enum {
  KSP_CONVERGED_RTOL = 2,
  KSP_CONVERGED_ATOL = 3,
  KSP_CONVERGED_ITS = 4,
  KSP_CONVERGED_HAPPY_BREAKDOWN = 7,
  KSP_CONVERGED_ITERATING = 0,
  KSP_DIVERGED_ITS = -3,
  KSP_DIVERGED_DTOL = -4,
  KSP_DIVERGED_BREAKDOWN = -5,
  KSP_DIVERGED_INDEFINITE_PC = -8,
  KSP_DIVERGED_NANORINF = -9,
  KSP_DIVERGED_INDEFINITE_MAT = -10
} KSPConvergedReason;

#endif /* FREHG_SHIM_PETSCKSP_H */
