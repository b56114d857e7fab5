/*
 * Sequential PETSc subset: the Vec/Mat calls the SNES residual and tangent
 * callbacks make, with PETSc 3.7 names, signatures and semantics.
 *
 * What the element-assembly path needs from PETSc (IGAP4STANDARD
 * src/snesiga_Residual.c, src/snesiga_Tangent.c, src/snesiga_init.c):
 *   - Vec: VecCreateMPI/VecDuplicate (one rank => sequential), array access,
 *     VecSet, VecSetValues with ADD_VALUES / INSERT_VALUES (written through
 *     immediately, so the last INSERT of a row wins), VecAssemblyBegin/End.
 *   - Mat: MatCreateAIJ with per-row preallocation, MatSetValues(ADD/INSERT)
 *     that inserts explicit zeros into the pattern (PETSc default),
 *     MatAssemblyBegin/End(FINAL) that compresses to CSR with ascending
 *     column indices, MatZeroEntries (values only), MatZeroRowsColumns with
 *     a diagonal value, MatSeqAIJGetArray / MatGetRowIJ for direct CSR access.
 * The KSP/SNES solver objects are not part of the assembly path; only the
 * SNES handle type exists here (the callbacks ignore it).
 *
 * A build against a real PETSc puts the real petscsnes.h first on the
 * include path; the callback code uses no call that is not in PETSc 3.7.
 */
#ifndef IGAB_PETSC_SUBSET_H
#define IGAB_PETSC_SUBSET_H

#include <stddef.h>
#include "mpi.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef int    PetscErrorCode;
typedef int    PetscInt;
typedef double PetscScalar;
typedef double PetscReal;
typedef int    PetscBool;
#define PETSC_TRUE  1
#define PETSC_FALSE 0
#define PETSC_NULL  NULL
#define PETSC_DECIDE (-1)
#define PETSC_DEFAULT (-2)

typedef struct _p_Vec  *Vec;
typedef struct _p_Mat  *Mat;
typedef struct _p_SNES *SNES;

typedef enum { NOT_SET_VALUES = 0, INSERT_VALUES = 1, ADD_VALUES = 2 } InsertMode;
typedef enum { MAT_FLUSH_ASSEMBLY = 1, MAT_FINAL_ASSEMBLY = 0 } MatAssemblyType;
typedef enum {
    MAT_KEEP_NONZERO_PATTERN = 1,
    MAT_NO_OFF_PROC_ZERO_ROWS = 2,
    MAT_SUBSET_OFF_PROC_ENTRIES = 3,
    MAT_SYMMETRIC = 4,
    MAT_SYMMETRY_ETERNAL = 5,
    MAT_NEW_NONZERO_ALLOCATION_ERR = 6,
    MAT_IGNORE_ZERO_ENTRIES = 7
} MatOption;

/* error codes (PETSc numbering for the few this subset raises) */
#define PETSC_ERR_MEM   55
#define PETSC_ERR_ARG_OUTOFRANGE 63
#define PETSC_ERR_ARG_WRONGSTATE 73
#define PETSC_ERR_LIB   76

/* ---- Vec ---- */
PetscErrorCode VecCreateSeq(MPI_Comm comm, PetscInt n, Vec *v);
PetscErrorCode VecCreateMPI(MPI_Comm comm, PetscInt n, PetscInt N, Vec *v);
PetscErrorCode VecDuplicate(Vec v, Vec *newv);
PetscErrorCode VecDestroy(Vec *v);
PetscErrorCode VecGetSize(Vec v, PetscInt *N);
PetscErrorCode VecGetLocalSize(Vec v, PetscInt *n);
PetscErrorCode VecGetArray(Vec v, PetscScalar **a);
PetscErrorCode VecRestoreArray(Vec v, PetscScalar **a);
PetscErrorCode VecGetArrayRead(Vec v, const PetscScalar **a);
PetscErrorCode VecRestoreArrayRead(Vec v, const PetscScalar **a);
PetscErrorCode VecSet(Vec v, PetscScalar alpha);
PetscErrorCode VecSetValues(Vec v, PetscInt n, const PetscInt idx[], const PetscScalar y[], InsertMode mode);
PetscErrorCode VecAssemblyBegin(Vec v);
PetscErrorCode VecAssemblyEnd(Vec v);
PetscErrorCode VecNorm2(Vec v, PetscReal *nrm);   /* subset helper: 2-norm */

/* ---- Mat (sequential AIJ) ---- */
PetscErrorCode MatCreateAIJ(MPI_Comm comm, PetscInt m, PetscInt n, PetscInt M, PetscInt N,
                            PetscInt d_nz, const PetscInt d_nnz[], PetscInt o_nz, const PetscInt o_nnz[], Mat *A);
PetscErrorCode MatCreateSeqAIJ(MPI_Comm comm, PetscInt m, PetscInt n, PetscInt nz, const PetscInt nnz[], Mat *A);
PetscErrorCode MatDestroy(Mat *A);
PetscErrorCode MatSetOption(Mat A, MatOption op, PetscBool flg);
PetscErrorCode MatGetSize(Mat A, PetscInt *m, PetscInt *n);
PetscErrorCode MatZeroEntries(Mat A);
PetscErrorCode MatSetValues(Mat A, PetscInt m, const PetscInt idxm[], PetscInt n, const PetscInt idxn[],
                            const PetscScalar v[], InsertMode mode);
PetscErrorCode MatAssemblyBegin(Mat A, MatAssemblyType type);
PetscErrorCode MatAssemblyEnd(Mat A, MatAssemblyType type);
PetscErrorCode MatAssembled(Mat A, PetscBool *assembled);
PetscErrorCode MatZeroRowsColumns(Mat A, PetscInt numRows, const PetscInt rows[], PetscScalar diag, Vec x, Vec b);
PetscErrorCode MatSeqAIJGetArray(Mat A, PetscScalar **array);
PetscErrorCode MatSeqAIJRestoreArray(Mat A, PetscScalar **array);
PetscErrorCode MatGetRowIJ(Mat A, PetscInt shift, PetscBool symmetric, PetscBool inodecompressed,
                           PetscInt *n, const PetscInt *ia[], const PetscInt *ja[], PetscBool *done);
PetscErrorCode MatRestoreRowIJ(Mat A, PetscInt shift, PetscBool symmetric, PetscBool inodecompressed,
                               PetscInt *n, const PetscInt *ia[], const PetscInt *ja[], PetscBool *done);
PetscErrorCode MatMult(Mat A, Vec x, Vec y);

#ifdef __cplusplus
}
#endif

#endif
