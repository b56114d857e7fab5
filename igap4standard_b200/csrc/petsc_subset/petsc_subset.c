/*
 * Sequential PETSc/MPI subset used where no PETSc or MPI is installed.
 *
 * Semantics follow PETSc 3.7 for the calls the SNES assembly callbacks make
 * (see petscsnes.h).  Errors are reported the PETSc way, by a nonzero
 * PetscErrorCode, and are also latched in the object (`err`) and printed once
 * to stderr, because the callbacks of IGAP4STANDARD ignore return codes
 * (src/snesiga_Residual.c:173, src/snesiga_Tangent.c:189): a silent error
 * there would turn into a wrong matrix, so the harness checks the latch.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include "petscsnes.h"

/* =========================================================== MPI (1 rank) */

#define MAILBOX_MAX 4096
typedef struct { int used; int tag; int bytes; void *data; } mail_t;
typedef struct { int used; int tag; int bytes; void *buf; } pending_t;
static mail_t    g_mail[MAILBOX_MAX];
static pending_t g_pend[MAILBOX_MAX];

static int type_size(MPI_Datatype t)
{
    switch (t) {
    case MPI_INT: return (int)sizeof(int);
    case MPI_DOUBLE: return (int)sizeof(double);
    case MPI_CHAR: return 1;
    default: return 0;
    }
}

int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return MPI_SUCCESS; }
int MPI_Finalize(void) { return MPI_SUCCESS; }
int MPI_Comm_size(MPI_Comm comm, int *size) { (void)comm; *size = 1; return MPI_SUCCESS; }
int MPI_Comm_rank(MPI_Comm comm, int *rank) { (void)comm; *rank = 0; return MPI_SUCCESS; }
int MPI_Barrier(MPI_Comm comm) { (void)comm; return MPI_SUCCESS; }

/* A message to self is copied at send time and matched by tag at MPI_Wait. */
int MPI_Isend(const void *buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm, MPI_Request *req)
{
    (void)comm;
    if (dest != 0) return MPI_ERR_OTHER;
    int bytes = count * type_size(type);
    for (int i = 0; i < MAILBOX_MAX; i++) {
        if (!g_mail[i].used) {
            g_mail[i].used = 1; g_mail[i].tag = tag; g_mail[i].bytes = bytes;
            g_mail[i].data = malloc(bytes > 0 ? (size_t)bytes : 1);
            if (bytes > 0) memcpy(g_mail[i].data, buf, (size_t)bytes);
            *req = -1;   /* sends complete immediately */
            return MPI_SUCCESS;
        }
    }
    return MPI_ERR_OTHER;
}

int MPI_Irecv(void *buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm comm, MPI_Request *req)
{
    (void)comm;
    if (source != 0) return MPI_ERR_OTHER;
    for (int i = 0; i < MAILBOX_MAX; i++) {
        if (!g_pend[i].used) {
            g_pend[i].used = 1; g_pend[i].tag = tag; g_pend[i].bytes = count * type_size(type); g_pend[i].buf = buf;
            *req = i;
            return MPI_SUCCESS;
        }
    }
    return MPI_ERR_OTHER;
}

int MPI_Wait(MPI_Request *req, MPI_Status *status)
{
    if (status) { status->MPI_SOURCE = 0; status->MPI_ERROR = MPI_SUCCESS; }
    if (*req < 0) return MPI_SUCCESS;
    pending_t *p = &g_pend[*req];
    for (int i = 0; i < MAILBOX_MAX; i++) {
        if (g_mail[i].used && g_mail[i].tag == p->tag) {
            if (g_mail[i].bytes != p->bytes) return MPI_ERR_OTHER;
            if (p->bytes > 0) memcpy(p->buf, g_mail[i].data, (size_t)p->bytes);
            free(g_mail[i].data);
            g_mail[i].used = 0;
            p->used = 0;
            if (status) status->MPI_TAG = p->tag;
            *req = -1;
            return MPI_SUCCESS;
        }
    }
    return MPI_ERR_OTHER;   /* no matching send on a single rank: a real MPI would hang */
}

int MPI_Gather(const void *sbuf, int scount, MPI_Datatype stype, void *rbuf, int rcount, MPI_Datatype rtype, int root, MPI_Comm comm)
{
    (void)rcount; (void)rtype; (void)root; (void)comm;
    memcpy(rbuf, sbuf, (size_t)scount * (size_t)type_size(stype));
    return MPI_SUCCESS;
}

int MPI_Gatherv(const void *sbuf, int scount, MPI_Datatype stype, void *rbuf, const int *rcounts, const int *displs, MPI_Datatype rtype, int root, MPI_Comm comm)
{
    (void)rcounts; (void)root; (void)comm;
    memcpy((char *)rbuf + (size_t)displs[0] * (size_t)type_size(rtype), sbuf, (size_t)scount * (size_t)type_size(stype));
    return MPI_SUCCESS;
}

int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root, MPI_Comm comm)
{
    (void)buf; (void)count; (void)type; (void)root; (void)comm;
    return MPI_SUCCESS;
}

int MPI_Scatter(const void *sbuf, int scount, MPI_Datatype stype, void *rbuf, int rcount, MPI_Datatype rtype, int root, MPI_Comm comm)
{
    (void)scount; (void)root; (void)comm;
    memcpy(rbuf, sbuf, (size_t)rcount * (size_t)type_size(rtype));
    (void)stype;
    return MPI_SUCCESS;
}

int MPI_Scatterv(const void *sbuf, const int *scounts, const int *displs, MPI_Datatype stype, void *rbuf, int rcount, MPI_Datatype rtype, int root, MPI_Comm comm)
{
    (void)scounts; (void)root; (void)comm; (void)rtype;
    memcpy(rbuf, (const char *)sbuf + (size_t)displs[0] * (size_t)type_size(stype), (size_t)rcount * (size_t)type_size(stype));
    return MPI_SUCCESS;
}

int MPI_Allreduce(const void *sbuf, void *rbuf, int count, MPI_Datatype type, MPI_Op op, MPI_Comm comm)
{
    (void)op; (void)comm;
    memmove(rbuf, sbuf, (size_t)count * (size_t)type_size(type));
    return MPI_SUCCESS;
}

/* =========================================================== Vec */

struct _p_Vec {
    PetscInt n;
    PetscScalar *a;
    int err;
};

static PetscErrorCode report(int *latch, PetscErrorCode code, const char *what)
{
    if (latch && !*latch) fprintf(stderr, "petsc_subset: error %d: %s\n", code, what);
    if (latch) *latch = code;
    return code;
}

PetscErrorCode VecCreateSeq(MPI_Comm comm, PetscInt n, Vec *v)
{
    (void)comm;
    Vec x = (Vec)calloc(1, sizeof(struct _p_Vec));
    if (!x) return PETSC_ERR_MEM;
    x->n = n;
    x->a = (PetscScalar *)calloc(n > 0 ? (size_t)n : 1, sizeof(PetscScalar));
    if (!x->a) { free(x); return PETSC_ERR_MEM; }
    *v = x;
    return 0;
}

PetscErrorCode VecCreateMPI(MPI_Comm comm, PetscInt n, PetscInt N, Vec *v)
{
    if (N >= 0 && N != n) return PETSC_ERR_ARG_OUTOFRANGE;   /* one rank owns everything */
    return VecCreateSeq(comm, n, v);
}

PetscErrorCode VecDuplicate(Vec v, Vec *newv) { return VecCreateSeq(MPI_COMM_SELF, v->n, newv); }

PetscErrorCode VecDestroy(Vec *v)
{
    if (v && *v) { free((*v)->a); free(*v); *v = NULL; }
    return 0;
}

PetscErrorCode VecGetSize(Vec v, PetscInt *N) { *N = v->n; return 0; }
PetscErrorCode VecGetLocalSize(Vec v, PetscInt *n) { *n = v->n; return 0; }
PetscErrorCode VecGetArray(Vec v, PetscScalar **a) { *a = v->a; return 0; }
PetscErrorCode VecRestoreArray(Vec v, PetscScalar **a) { (void)v; *a = NULL; return 0; }
PetscErrorCode VecGetArrayRead(Vec v, const PetscScalar **a) { *a = v->a; return 0; }
PetscErrorCode VecRestoreArrayRead(Vec v, const PetscScalar **a) { (void)v; *a = NULL; return 0; }

PetscErrorCode VecSet(Vec v, PetscScalar alpha)
{
    for (PetscInt i = 0; i < v->n; i++) v->a[i] = alpha;
    return 0;
}

PetscErrorCode VecSetValues(Vec v, PetscInt n, const PetscInt idx[], const PetscScalar y[], InsertMode mode)
{
    for (PetscInt k = 0; k < n; k++) {
        PetscInt i = idx[k];
        if (i < 0) continue;                       /* PETSc ignores negative indices */
        if (i >= v->n) return report(&v->err, PETSC_ERR_ARG_OUTOFRANGE, "VecSetValues index out of range");
        if (mode == ADD_VALUES) v->a[i] += y[k]; else v->a[i] = y[k];
    }
    return 0;
}

PetscErrorCode VecAssemblyBegin(Vec v) { (void)v; return 0; }
PetscErrorCode VecAssemblyEnd(Vec v) { (void)v; return 0; }

PetscErrorCode VecNorm2(Vec v, PetscReal *nrm)
{
    double s = 0.0;
    for (PetscInt i = 0; i < v->n; i++) s += v->a[i] * v->a[i];
    *nrm = sqrt(s);
    return 0;
}

/* =========================================================== Mat (seq AIJ) */

struct _p_Mat {
    PetscInt m, n;
    PetscInt *start;     /* [m+1] row start in storage */
    PetscInt *len;       /* [m]   used entries per row */
    PetscInt *cols;      /* storage, ascending per row */
    PetscScalar *vals;
    int assembled;       /* storage compressed to CSR */
    int ignore_zero;
    int err;
};

PetscErrorCode MatCreateSeqAIJ(MPI_Comm comm, PetscInt m, PetscInt n, PetscInt nz, const PetscInt nnz[], Mat *A)
{
    (void)comm;
    Mat M = (Mat)calloc(1, sizeof(struct _p_Mat));
    if (!M) return PETSC_ERR_MEM;
    M->m = m; M->n = n;
    M->start = (PetscInt *)malloc(((size_t)m + 1) * sizeof(PetscInt));
    M->len = (PetscInt *)calloc(m > 0 ? (size_t)m : 1, sizeof(PetscInt));
    if (!M->start || !M->len) { free(M->start); free(M->len); free(M); return PETSC_ERR_MEM; }
    size_t total = 0;
    M->start[0] = 0;
    for (PetscInt r = 0; r < m; r++) {
        PetscInt c = nnz ? nnz[r] : nz;
        if (c < 0) c = 0;
        if (c > n) c = n;
        total += (size_t)c;
        if (total > 2147483647u) { free(M->start); free(M->len); free(M); return PETSC_ERR_ARG_OUTOFRANGE; }
        M->start[r + 1] = (PetscInt)total;
    }
    M->cols = (PetscInt *)malloc((total > 0 ? total : 1) * sizeof(PetscInt));
    M->vals = (PetscScalar *)calloc(total > 0 ? total : 1, sizeof(PetscScalar));
    if (!M->cols || !M->vals) { free(M->cols); free(M->vals); free(M->start); free(M->len); free(M); return PETSC_ERR_MEM; }
    *A = M;
    return 0;
}

/* One rank: the diagonal and off-diagonal preallocations add up (src/snesiga_init.c:360). */
PetscErrorCode MatCreateAIJ(MPI_Comm comm, PetscInt m, PetscInt n, PetscInt M, PetscInt N,
                            PetscInt d_nz, const PetscInt d_nnz[], PetscInt o_nz, const PetscInt o_nnz[], Mat *A)
{
    if ((M >= 0 && M != m) || (N >= 0 && N != n)) return PETSC_ERR_ARG_OUTOFRANGE;
    PetscInt *nnz = (PetscInt *)malloc((m > 0 ? (size_t)m : 1) * sizeof(PetscInt));
    if (!nnz) return PETSC_ERR_MEM;
    for (PetscInt r = 0; r < m; r++)
        nnz[r] = (d_nnz ? d_nnz[r] : d_nz) + (o_nnz ? o_nnz[r] : (o_nz > 0 ? o_nz : 0));
    PetscErrorCode e = MatCreateSeqAIJ(comm, m, n, 0, nnz, A);
    free(nnz);
    return e;
}

PetscErrorCode MatDestroy(Mat *A)
{
    if (A && *A) {
        free((*A)->start); free((*A)->len); free((*A)->cols); free((*A)->vals); free(*A);
        *A = NULL;
    }
    return 0;
}

PetscErrorCode MatSetOption(Mat A, MatOption op, PetscBool flg)
{
    if (op == MAT_IGNORE_ZERO_ENTRIES) A->ignore_zero = flg;
    return 0;
}

PetscErrorCode MatGetSize(Mat A, PetscInt *m, PetscInt *n) { if (m) *m = A->m; if (n) *n = A->n; return 0; }

PetscErrorCode MatZeroEntries(Mat A)
{
    memset(A->vals, 0, (size_t)A->start[A->m] * sizeof(PetscScalar));
    return 0;
}

static PetscErrorCode mat_set_one(Mat A, PetscInt r, PetscInt c, PetscScalar v, InsertMode mode)
{
    PetscInt *cols = A->cols + A->start[r];
    PetscScalar *vals = A->vals + A->start[r];
    PetscInt lo = 0, hi = A->len[r];
    while (lo < hi) {
        PetscInt mid = (lo + hi) >> 1;
        if (cols[mid] < c) lo = mid + 1; else hi = mid;
    }
    if (lo < A->len[r] && cols[lo] == c) {
        if (mode == ADD_VALUES) vals[lo] += v; else vals[lo] = v;
        return 0;
    }
    if (A->ignore_zero && v == 0.0) return 0;
    PetscInt cap = A->start[r + 1] - A->start[r];
    if (A->len[r] >= cap)
        return report(&A->err, PETSC_ERR_ARG_OUTOFRANGE, "MatSetValues: new nonzero beyond the preallocation");
    for (PetscInt k = A->len[r]; k > lo; k--) { cols[k] = cols[k - 1]; vals[k] = vals[k - 1]; }
    cols[lo] = c;
    vals[lo] = v;
    A->len[r]++;
    return 0;
}

PetscErrorCode MatSetValues(Mat A, PetscInt m, const PetscInt idxm[], PetscInt n, const PetscInt idxn[],
                            const PetscScalar v[], InsertMode mode)
{
    for (PetscInt i = 0; i < m; i++) {
        PetscInt r = idxm[i];
        if (r < 0) continue;
        if (r >= A->m) return report(&A->err, PETSC_ERR_ARG_OUTOFRANGE, "MatSetValues row out of range");
        for (PetscInt j = 0; j < n; j++) {
            PetscInt c = idxn[j];
            if (c < 0) continue;
            if (c >= A->n) return report(&A->err, PETSC_ERR_ARG_OUTOFRANGE, "MatSetValues column out of range");
            PetscErrorCode e = mat_set_one(A, r, c, v[(size_t)i * (size_t)n + (size_t)j], mode);
            if (e) return e;
        }
    }
    return 0;
}

PetscErrorCode MatAssemblyBegin(Mat A, MatAssemblyType type) { (void)A; (void)type; return 0; }

/* FINAL assembly squeezes the unused preallocation out, as MatAssemblyEnd_SeqAIJ does. */
PetscErrorCode MatAssemblyEnd(Mat A, MatAssemblyType type)
{
    if (type != MAT_FINAL_ASSEMBLY) return 0;
    PetscInt w = 0;
    for (PetscInt r = 0; r < A->m; r++) {
        PetscInt s = A->start[r], l = A->len[r];
        if (s != w) {
            memmove(A->cols + w, A->cols + s, (size_t)l * sizeof(PetscInt));
            memmove(A->vals + w, A->vals + s, (size_t)l * sizeof(PetscScalar));
        }
        A->start[r] = w;
        w += l;
    }
    A->start[A->m] = w;
    A->assembled = 1;
    return 0;
}

PetscErrorCode MatAssembled(Mat A, PetscBool *assembled) { *assembled = A->assembled; return 0; }

/* Zero the listed rows and the same columns, put `diag` on the diagonal of each
 * listed row; with x and b given, also b_rows = diag*x_rows and
 * b_other -= A(other, rows)*x_rows (PETSc MatZeroRowsColumns semantics). */
PetscErrorCode MatZeroRowsColumns(Mat A, PetscInt numRows, const PetscInt rows[], PetscScalar diag, Vec x, Vec b)
{
    if (A->m != A->n) return report(&A->err, PETSC_ERR_ARG_WRONGSTATE, "MatZeroRowsColumns needs a square matrix");
    char *mask = (char *)calloc(A->m > 0 ? (size_t)A->m : 1, 1);
    if (!mask) return PETSC_ERR_MEM;
    for (PetscInt k = 0; k < numRows; k++) {
        PetscInt r = rows[k];
        if (r < 0 || r >= A->m) { free(mask); return report(&A->err, PETSC_ERR_ARG_OUTOFRANGE, "MatZeroRowsColumns row out of range"); }
        mask[r] = 1;
    }
    if (x && b) {
        for (PetscInt r = 0; r < A->m; r++) {
            if (mask[r]) continue;
            for (PetscInt k = A->start[r]; k < A->start[r] + A->len[r]; k++)
                if (mask[A->cols[k]]) b->a[r] -= A->vals[k] * x->a[A->cols[k]];
        }
        for (PetscInt r = 0; r < A->m; r++) if (mask[r]) b->a[r] = diag * x->a[r];
    }
    for (PetscInt r = 0; r < A->m; r++) {
        for (PetscInt k = A->start[r]; k < A->start[r] + A->len[r]; k++)
            if (mask[r] || mask[A->cols[k]]) A->vals[k] = 0.0;
    }
    PetscErrorCode e = 0;
    for (PetscInt r = 0; r < A->m && !e; r++) {
        if (!mask[r]) continue;
        e = mat_set_one(A, r, r, diag, INSERT_VALUES);
    }
    free(mask);
    return e;
}

PetscErrorCode MatSeqAIJGetArray(Mat A, PetscScalar **array) { *array = A->vals; return 0; }
PetscErrorCode MatSeqAIJRestoreArray(Mat A, PetscScalar **array) { (void)A; *array = NULL; return 0; }

PetscErrorCode MatGetRowIJ(Mat A, PetscInt shift, PetscBool symmetric, PetscBool inodecompressed,
                           PetscInt *n, const PetscInt *ia[], const PetscInt *ja[], PetscBool *done)
{
    (void)symmetric; (void)inodecompressed;
    if (!A->assembled || shift != 0) { *done = PETSC_FALSE; return 0; }
    *n = A->m; *ia = A->start; *ja = A->cols; *done = PETSC_TRUE;
    return 0;
}

PetscErrorCode MatRestoreRowIJ(Mat A, PetscInt shift, PetscBool symmetric, PetscBool inodecompressed,
                               PetscInt *n, const PetscInt *ia[], const PetscInt *ja[], PetscBool *done)
{
    (void)A; (void)shift; (void)symmetric; (void)inodecompressed; (void)n;
    *ia = NULL; *ja = NULL; *done = PETSC_TRUE;
    return 0;
}

PetscErrorCode MatMult(Mat A, Vec x, Vec y)
{
    for (PetscInt r = 0; r < A->m; r++) {
        double s = 0.0;
        for (PetscInt k = A->start[r]; k < A->start[r] + A->len[r]; k++) s += A->vals[k] * x->a[A->cols[k]];
        y->a[r] = s;
    }
    return 0;
}

/* ---- subset-only introspection used by test harnesses ---- */
int petsc_subset_mat_error(Mat A) { return A->err; }
int petsc_subset_vec_error(Vec v) { return v->err; }
