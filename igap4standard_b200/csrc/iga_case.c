/*
 * Single-rank case builder (see include/iga_case.h).
 *
 * One rank, p = 2 (mesh/nurbs/nurbs_init.c with npart = {1,1,1}, ipart = 0): the
 * faces of the non-periodic directions are the boundaries (:24-27), the rank owns
 * nelem + 2 points along a non-periodic direction and nelem along a periodic one
 * (:36-39), and along every periodic direction it is its own neighbour: the halo
 * parts of set_mpi_part (:156-199) are all rank 0, so the ghost layers arrive as
 * messages to self.  The universal index of an owned point follows :42-47.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "igap4_structs.h"
#include "iga_case.h"

/* whichever library this file is linked into provides these */
void snesiga_init(void *app_, void *phys_, void *nurbs_, void *bc_, void *snesassmbl_, void *iocomm_);
/* present only in libsnesiga_b200: lets the GPU callbacks call the case's hook */
extern int snesiga_gpu_set_neumann(void *app_, void (*fn)(double *, double[], int, int, int, double[])) __attribute__((weak));
/* the reference's CPU integrands, present only when linked for the oracle */
extern void ge_residual(double *, double *, double *) __attribute__((weak));
extern void ge_tangent(double *, double *, double *) __attribute__((weak));
extern void getime_residual(double *, double *, double *) __attribute__((weak));
extern void getime_tangent(double *, double *, double *) __attribute__((weak));
extern void ge_density(double *, double *, double *) __attribute__((weak));
extern void ge_densityb(double *, double *, double, double *, int) __attribute__((weak));
extern void getime_density(double *, double *, double *) __attribute__((weak));
extern void getime_densityb(double *, double *, double, double *, int) __attribute__((weak));
/* the solver loop (present in libsnesiga_b200: the device Newton solve) */
extern void snes_solve(void *snesassmbl_) __attribute__((weak));
/* subset-only error latches (weak: absent under a real PETSc) */
extern int petsc_subset_mat_error(Mat A) __attribute__((weak));
extern int petsc_subset_vec_error(Vec v) __attribute__((weak));

#define NPAR_NEUMANN_MIN 39

struct iga_case {
    Phys phys;
    Nurbs nurbs;
    BC bc;
    IGA app;
    SNESAssmbl sa;
    IOcomm io;
    int kind;
    int ndof;
    int n_par_neumann;
};

void iga_case_neumann(double *neumann_, double par_neumann[], int face_id, int bc_order, int idof, double xq[])
{
    double s = 1.0 + par_neumann[36] * xq[0] + par_neumann[37] * xq[1] + par_neumann[38] * xq[2];
    *neumann_ = par_neumann[6 * face_id + 3 * bc_order + idof] * s;
}

/* The app hook of the reference's library interface (include/bc.h:14).  An
 * application that defines its own `neumann` overrides this one. */
__attribute__((weak)) void neumann(double *neumann_, double par_neumann[], int face_id, int bc_order, int idof, double xq[])
{
    iga_case_neumann(neumann_, par_neumann, face_id, bc_order, idof, xq);
}

static void *xmalloc(size_t n) { return malloc(n > 0 ? n : 1); }

iga_case *iga_case_create(int phys_kind, const int nelem[3], const double *knots,
                          const double par_mat[9], const int bc_type[36],
                          const double par_periodic[9], const double par_dirichlet[9],
                          const double *par_neumann, int n_par_neumann)
{
    const int none[3] = {0, 0, 0};
    return iga_case_create_periodic(phys_kind, nelem, knots, par_mat, bc_type, par_periodic, par_dirichlet,
                                    par_neumann, n_par_neumann, none);
}

/* the halo parts of one rank that is its own neighbour along the periodic directions:
 * blocks 0-6 = z, y, x, yz, xz, xy, xyz in set_mpi_part's order (nurbs_init.c:162-169) */
static int self_blocks(const int per[3], int *block)
{
    const int c0 = per[0], c1 = per[1], c2 = per[2];
    const int on[7] = {c2, c1, c0, c1 && c2, c0 && c2, c0 && c1, c0 && c1 && c2};
    int n = 0;
    for (int b = 0; b < 7; b++)
        if (on[b]) {
            if (block) block[n] = b;
            n++;
        }
    return n;
}

iga_case *iga_case_create_periodic(int phys_kind, const int nelem[3], const double *knots,
                                   const double par_mat[9], const int bc_type[36],
                                   const double par_periodic[9], const double par_dirichlet[9],
                                   const double *par_neumann, int n_par_neumann, const int bc_periodic[3])
{
    const int p = 2;
    if (phys_kind != IGA_CASE_GE && phys_kind != IGA_CASE_GETIME) return NULL;
    for (int d = 0; d < 3; d++) if (nelem[d] < 1) return NULL;
    for (int d = 0; d < 3; d++)
        if ((bc_periodic[d] != 0 && bc_periodic[d] != 1) || (bc_periodic[d] && nelem[d] < 3)) return NULL;
    iga_case *c = (iga_case *)calloc(1, sizeof(iga_case));
    if (!c) return NULL;
    c->kind = phys_kind;

    /* ---- Phys (phys/ge/init.c:10-15, phys/getime/init.c:10-15) */
    c->phys.ndim = 3;
    c->phys.ndof = 3;
    c->phys.torder = (phys_kind == IGA_CASE_GE) ? 0 : 2;
    c->phys.sorder = 2;
    c->phys.ndensity = (phys_kind == IGA_CASE_GE) ? 13 : 2;
    c->phys.nfield = (phys_kind == IGA_CASE_GE) ? 33 : 6;
    c->phys.par_mat = (double *)xmalloc(9 * sizeof(double));
    memcpy(c->phys.par_mat, par_mat, 9 * sizeof(double));
    c->phys.residual = (phys_kind == IGA_CASE_GE) ? ge_residual : getime_residual;
    c->phys.tangent = (phys_kind == IGA_CASE_GE) ? ge_tangent : getime_tangent;
    c->phys.density = (phys_kind == IGA_CASE_GE) ? ge_density : getime_density;
    c->phys.densityb = (phys_kind == IGA_CASE_GE) ? ge_densityb : getime_densityb;

    /* ---- Nurbs, one rank */
    Nurbs *nb = &c->nurbs;
    nb->porder = p;
    nb->nelem = (int *)xmalloc(3 * sizeof(int));
    nb->nbasis = (int *)xmalloc(3 * sizeof(int));
    nb->nknot = (int *)xmalloc(3 * sizeof(int));
    nb->knotVector = (double **)xmalloc(3 * sizeof(double *));
    size_t off = 0;
    for (int d = 0; d < 3; d++) {
        nb->nelem[d] = nelem[d];
        nb->nbasis[d] = bc_periodic[d] ? nelem[d] : nelem[d] + p;
        nb->nknot[d] = nelem[d] + 1 + 2 * p;
        nb->knotVector[d] = (double *)xmalloc((size_t)nb->nknot[d] * sizeof(double));
        memcpy(nb->knotVector[d], knots + off, (size_t)nb->nknot[d] * sizeof(double));
        off += (size_t)nb->nknot[d];
    }
    nb->nboun = 0;
    nb->boun = (int *)xmalloc(6 * sizeof(int));
    for (int f = 0; f < 6; f++)
        if (!bc_periodic[f / 2]) nb->boun[nb->nboun++] = f;
    const int npart = self_blocks(bc_periodic, NULL);
    nb->nsendPart = npart;
    nb->sendPart = (int *)calloc((size_t)(npart > 0 ? npart : 1), sizeof(int));   /* rank 0: itself */
    nb->nrecvPart = npart;
    nb->recvPart = (int *)calloc((size_t)(npart > 0 ? npart : 1), sizeof(int));
    nb->sendBlock = (int *)xmalloc((size_t)npart * sizeof(int));
    nb->recvBlock = (int *)xmalloc((size_t)npart * sizeof(int));
    self_blocks(bc_periodic, nb->sendBlock);
    self_blocks(bc_periodic, nb->recvBlock);
    int ncp = nb->nbasis[0] * nb->nbasis[1] * nb->nbasis[2];
    nb->universalIdx_temp = (int *)xmalloc((size_t)ncp * sizeof(int));
    {
        const int gy = nelem[1] + (bc_periodic[1] ? 0 : p), gz = nelem[2] + (bc_periodic[2] ? 0 : p);
        int ia = 0;
        for (int x = 0; x < nb->nbasis[0]; x++)
            for (int y = 0; y < nb->nbasis[1]; y++)
                for (int z = 0; z < nb->nbasis[2]; z++) nb->universalIdx_temp[ia++] = gy * gz * x + gz * y + z;
    }
    nb->bc_periodic = NULL;
    nb->nelem_global = NULL;
    nb->knotVector_global = NULL;

    /* ---- BC */
    c->bc.bc_type = (int *)xmalloc(36 * sizeof(int));
    memcpy(c->bc.bc_type, bc_type, 36 * sizeof(int));
    c->bc.par_periodic = (double *)xmalloc(9 * sizeof(double));
    memcpy(c->bc.par_periodic, par_periodic, 9 * sizeof(double));
    c->bc.par_dirichlet = (double *)xmalloc(9 * sizeof(double));
    memcpy(c->bc.par_dirichlet, par_dirichlet, 9 * sizeof(double));
    int npn = n_par_neumann > NPAR_NEUMANN_MIN ? n_par_neumann : NPAR_NEUMANN_MIN;
    c->bc.par_neumann = (double *)calloc((size_t)npn, sizeof(double));
    if (par_neumann && n_par_neumann > 0) memcpy(c->bc.par_neumann, par_neumann, (size_t)n_par_neumann * sizeof(double));
    c->n_par_neumann = npn;

    /* ---- IGA + SNES objects (src/snesiga_init.c:12-132) */
    snesiga_init(&c->app, &c->phys, &c->nurbs, &c->bc, &c->sa, &c->io);
    c->ndof = c->app.nselfIdx;
    if (snesiga_gpu_set_neumann) snesiga_gpu_set_neumann(&c->app, neumann);
    return c;
}

extern int snesiga_gpu_free(void *app_) __attribute__((weak));

void iga_case_destroy(iga_case *c)
{
    if (!c) return;
    /* the GPU state is keyed by the IGA address, which a later case may reuse */
    if (snesiga_gpu_free) snesiga_gpu_free(&c->app);
    VecDestroy(&c->sa.Residual_);
    VecDestroy(&c->sa.U);
    MatDestroy(&c->sa.Tangent_);
    free(c->app.selfIdx); free(c->app.sendIdx); free(c->app.sendPtr);
    free(c->app.recvIdx); free(c->app.recvPtr); free(c->app.globalIdx);
    free(c->app.U_hist);
    free(c->io.nDof_array); free(c->io.iDof_displ_array); free(c->io.universalIdx);
    for (int d = 0; d < 3; d++) free(c->nurbs.knotVector[d]);
    free(c->nurbs.knotVector); free(c->nurbs.nelem); free(c->nurbs.nbasis); free(c->nurbs.nknot);
    free(c->nurbs.boun); free(c->nurbs.sendPart); free(c->nurbs.recvPart);
    free(c->bc.bc_type); free(c->bc.par_periodic); free(c->bc.par_dirichlet); free(c->bc.par_neumann);
    free(c->phys.par_mat);
    free(c);
}

int iga_case_ndof(const iga_case *c) { return c->ndof; }

int iga_case_index_maps(const iga_case *c, int n[3], int *selfIdx, int *sendIdx, int *recvIdx, int *globalIdx)
{
    if (!c || !n) return -1;
    const IGA *a = &c->app;
    n[0] = a->nselfIdx;
    n[1] = a->nsendIdx;
    n[2] = a->nrecvIdx;
    if (selfIdx) memcpy(selfIdx, a->selfIdx, (size_t)a->nselfIdx * sizeof(int));
    if (sendIdx) memcpy(sendIdx, a->sendIdx, (size_t)a->nsendIdx * sizeof(int));
    if (recvIdx) memcpy(recvIdx, a->recvIdx, (size_t)a->nrecvIdx * sizeof(int));
    if (globalIdx) memcpy(globalIdx, a->globalIdx, (size_t)(a->nselfIdx + a->nrecvIdx) * sizeof(int));
    return 0;
}

int iga_case_set_history(iga_case *c, int level, const double *U)
{
    if (level < 0 || level > c->phys.torder) return 1;
    memcpy(c->app.U_hist + (size_t)level * (size_t)c->ndof, U, (size_t)c->ndof * sizeof(double));
    return 0;
}

int iga_case_get_history(const iga_case *c, int level, double *U)
{
    if (level < 0 || level > c->phys.torder) return 1;
    memcpy(U, c->app.U_hist + (size_t)level * (size_t)c->ndof, (size_t)c->ndof * sizeof(double));
    return 0;
}

int iga_case_set_par_neumann(iga_case *c, const double *par_neumann, int n)
{
    if (n > c->n_par_neumann) return 1;
    memcpy(c->bc.par_neumann, par_neumann, (size_t)n * sizeof(double));
    return 0;
}

int iga_case_set_par_dirichlet(iga_case *c, const double par_dirichlet[9])
{
    memcpy(c->bc.par_dirichlet, par_dirichlet, 9 * sizeof(double));
    return 0;
}

int iga_case_set_par_mat(iga_case *c, const double par_mat[9])
{
    memcpy(c->phys.par_mat, par_mat, 9 * sizeof(double));
    return 0;
}

static int latched(const iga_case *c)
{
    int e = 0;
    if (petsc_subset_vec_error) e = e ? e : petsc_subset_vec_error(c->sa.Residual_);
    if (petsc_subset_mat_error) e = e ? e : petsc_subset_mat_error(c->sa.Tangent_);
    return e;
}

int iga_case_residual(iga_case *c, const double *U, double *R)
{
    PetscScalar *u;
    VecGetArray(c->sa.U, &u);
    memcpy(u, U, (size_t)c->ndof * sizeof(double));
    VecRestoreArray(c->sa.U, &u);
    PetscErrorCode e = c->sa.snes_Residual(NULL, c->sa.U, c->sa.Residual_, &c->app);
    if (e) return e;
    const PetscScalar *r;
    VecGetArrayRead(c->sa.Residual_, &r);
    memcpy(R, r, (size_t)c->ndof * sizeof(double));
    VecRestoreArrayRead(c->sa.Residual_, &r);
    return latched(c);
}

int iga_case_tangent(iga_case *c, const double *U)
{
    PetscScalar *u;
    VecGetArray(c->sa.U, &u);
    memcpy(u, U, (size_t)c->ndof * sizeof(double));
    VecRestoreArray(c->sa.U, &u);
    PetscErrorCode e = c->sa.snes_Tangent(NULL, c->sa.U, c->sa.Tangent_, c->sa.Tangent_, &c->app);
    if (e) return e;
    return latched(c);
}

long iga_case_tangent_nnz(const iga_case *c)
{
    PetscInt n;
    const PetscInt *ia, *ja;
    PetscBool done;
    MatGetRowIJ(c->sa.Tangent_, 0, PETSC_FALSE, PETSC_FALSE, &n, &ia, &ja, &done);
    if (!done) return -1;
    long nnz = ia[n];
    MatRestoreRowIJ(c->sa.Tangent_, 0, PETSC_FALSE, PETSC_FALSE, &n, &ia, &ja, &done);
    return nnz;
}

int iga_case_tangent_csr(const iga_case *c, int *rowptr, int *cols, double *vals)
{
    PetscInt n;
    const PetscInt *ia, *ja;
    PetscBool done;
    MatGetRowIJ(c->sa.Tangent_, 0, PETSC_FALSE, PETSC_FALSE, &n, &ia, &ja, &done);
    if (!done) return 1;
    long nnz = ia[n];
    if (rowptr) memcpy(rowptr, ia, ((size_t)n + 1) * sizeof(int));
    if (cols) memcpy(cols, ja, (size_t)nnz * sizeof(int));
    MatRestoreRowIJ(c->sa.Tangent_, 0, PETSC_FALSE, PETSC_FALSE, &n, &ia, &ja, &done);
    if (vals) {
        PetscScalar *a;
        MatSeqAIJGetArray(c->sa.Tangent_, &a);
        memcpy(vals, a, (size_t)nnz * sizeof(double));
        MatSeqAIJRestoreArray(c->sa.Tangent_, &a);
    }
    return 0;
}

void *iga_case_app(iga_case *c) { return &c->app; }
void *iga_case_iocomm(iga_case *c) { return &c->io; }
void *iga_case_snesassmbl(iga_case *c) { return &c->sa; }

int iga_case_solve(iga_case *c, double *U)
{
    if (!snes_solve) return -1;
    PetscScalar *u;
    VecGetArray(c->sa.U, &u);
    memcpy(u, U, (size_t)c->ndof * sizeof(double));
    VecRestoreArray(c->sa.U, &u);
    c->sa.converged = 0;
    snes_solve(&c->sa);
    VecGetArray(c->sa.U, &u);
    memcpy(U, u, (size_t)c->ndof * sizeof(double));
    VecRestoreArray(c->sa.U, &u);
    return c->sa.converged ? 0 : 1;
}
