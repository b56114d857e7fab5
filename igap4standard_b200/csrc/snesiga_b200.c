/*
 * PETSc SNES callbacks on top of libigap4_b200 (include/snesiga_b200.h).
 *
 * Host C only: PETSc objects are read and written through their public API
 * (VecGetArrayRead, VecGetArray, MatSeqAIJGetArray, MatGetRowIJ), the
 * assembly itself happens on the GPU through the igab C ABI.
 */
#include <stdio.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include "petscsnes.h"
#include "igap4_structs.h"
#include "igab.h"
#include "snesiga_b200.h"

#ifndef PETSC_ERR_SUP
#define PETSC_ERR_SUP 56
#endif
#ifndef PETSC_ERR_FP
#define PETSC_ERR_FP 72
#endif
#ifndef PETSC_ERR_LIB
#define PETSC_ERR_LIB 76
#endif

/* the application's traction hook; weak so that the library loads without one */
extern void neumann(double *neumann_, double par_neumann[], int face_id, int bc_order, int idof, double xq[]) __attribute__((weak));

typedef void (*neumann_fn)(double *, double[], int, int, int, double[]);

typedef struct gpu_state {
    IGA *app;
    igab_ctx *ctx;
    int device;
    long ndof, nnz;
    neumann_fn nfn;
    int npol, nwatch, neu_done;
    double *nwatch_copy;
    long npts;
    double *nxyz;   /* 3 per point */
    int *nmeta;     /* face, order, dof per point */
    double *nval;
    Mat pattern_ok; /* last matrix whose pattern was checked */
    int prec;
    double *vals32; /* host widening buffer for the FP32 mode (floats) */
    double ms[4];
    double ksp_rtol;                 /* device Newton solve: Krylov tolerance (0: PETSc's default 1e-5) */
    int ksp_maxit;
    igab_newton_info last_solve;
    struct gpu_state *next;
} gpu_state;

/* which SNESAssmbl belongs to which IGA (recorded by snesiga_init; the reference's
 * snes_solve(void *snesassmbl) has no application argument) */
typedef struct sa_link {
    void *sa, *app;
    struct sa_link *next;
} sa_link;
static sa_link *g_links = NULL;

static void link_snesassmbl(void *sa, void *app)
{
    for (sa_link *l = g_links; l; l = l->next)
        if (l->sa == sa) { l->app = app; return; }
    sa_link *l = (sa_link *)malloc(sizeof(sa_link));
    if (!l) return;
    l->sa = sa;
    l->app = app;
    l->next = g_links;
    g_links = l;
}

static void *app_of_snesassmbl(void *sa)
{
    for (sa_link *l = g_links; l; l = l->next)
        if (l->sa == sa) return l->app;
    return NULL;
}

static gpu_state *g_states = NULL;

static double now_ms(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec * 1e3 + ts.tv_nsec * 1e-6;
}

static gpu_state *find_state(void *app)
{
    for (gpu_state *s = g_states; s; s = s->next)
        if (s->app == (IGA *)app) return s;
    return NULL;
}

static PetscErrorCode map_err(int rc)
{
    if (rc == IGAB_OK) return 0;
    if (rc == IGAB_ERR_NONFINITE) return PETSC_ERR_FP;
    if (rc == IGAB_ERR_UNSUPPORTED || rc == IGAB_ERR_ARG) return PETSC_ERR_SUP;
    if (rc == IGAB_ERR_NOMEM) return PETSC_ERR_MEM;
    return PETSC_ERR_LIB;
}

static int create_state(IGA *app, int device, gpu_state **out)
{
    Phys *phys = app->phys;
    Nurbs *nurbs = app->nurbs;
    BC *bc = app->bc;
    int nproc = 1;
    MPI_Comm_size(MPI_COMM_WORLD, &nproc);
    int self_only = nproc == 1;
    for (int i = 0; i < nurbs->nsendPart; i++) self_only = self_only && nurbs->sendPart[i] == 0;
    for (int i = 0; i < nurbs->nrecvPart; i++) self_only = self_only && nurbs->recvPart[i] == 0;
    if (!self_only) {
        fprintf(stderr, "snesiga_b200: only single-rank meshes are supported (periodic directions included)\n");
        return PETSC_ERR_SUP;
    }
    if (phys->ndim != 3 || phys->ndof != 3 || nurbs->porder != 2 || (phys->torder != 0 && phys->torder != 2)) {
        fprintf(stderr, "snesiga_b200: needs ndim = ndof = 3, porder = 2 and torder 0 (ge) or 2 (getime)\n");
        return PETSC_ERR_SUP;
    }
    igab_mesh_desc d;
    memset(&d, 0, sizeof(d));
    d.phys = phys->torder == 0 ? IGAB_PHYS_GE : IGAB_PHYS_GETIME;
    long nk = 0;
    for (int i = 0; i < 3; i++) { d.nelem[i] = nurbs->nelem[i]; nk += nurbs->nelem[i] + 5; }
    double *knots = (double *)malloc((size_t)nk * sizeof(double));
    if (!knots) return PETSC_ERR_MEM;
    long o = 0;
    for (int i = 0; i < 3; i++) {
        if (nurbs->nknot[i] != nurbs->nelem[i] + 5) { free(knots); return PETSC_ERR_SUP; }
        memcpy(knots + o, nurbs->knotVector[i], (size_t)nurbs->nknot[i] * sizeof(double));
        o += nurbs->nknot[i];
    }
    d.knots = knots;
    memcpy(d.par_mat, phys->par_mat, 9 * sizeof(double));
    memcpy(d.bc_type, bc->bc_type, 36 * sizeof(int));
    memcpy(d.par_periodic, bc->par_periodic, 9 * sizeof(double));
    memcpy(d.par_dirichlet, bc->par_dirichlet, 9 * sizeof(double));
    /* one rank: a direction whose owned points number its elements is periodic
     * (mesh/nurbs/nurbs_init.c:39) */
    for (int i = 0; i < 3; i++) d.bc_periodic[i] = nurbs->nbasis[i] == nurbs->nelem[i];
    gpu_state *s = (gpu_state *)calloc(1, sizeof(gpu_state));
    if (!s) { free(knots); return PETSC_ERR_MEM; }
    int rc = igab_create(&d, device, &s->ctx);
    free(knots);
    if (rc) {
        fprintf(stderr, "snesiga_b200: igab_create failed: %s\n", igab_last_error());
        free(s);
        return map_err(rc);
    }
    s->app = app;
    s->device = device;
    igab_sizes(s->ctx, &s->ndof, &s->nnz, NULL);
    if (s->ndof != app->nselfIdx) {
        fprintf(stderr, "snesiga_b200: dof count %ld does not match nselfIdx %d\n", s->ndof, app->nselfIdx);
        igab_destroy(s->ctx);
        free(s);
        return PETSC_ERR_SUP;
    }
    s->nfn = neumann;
    igab_neumann_points(s->ctx, &s->npts, NULL, NULL);
    if (s->npts > 0) {
        s->nxyz = (double *)malloc((size_t)s->npts * 3 * sizeof(double));
        s->nmeta = (int *)malloc((size_t)s->npts * 3 * sizeof(int));
        s->nval = (double *)malloc((size_t)s->npts * sizeof(double));
        if (!s->nxyz || !s->nmeta || !s->nval) { igab_destroy(s->ctx); free(s); return PETSC_ERR_MEM; }
        igab_neumann_points(s->ctx, &s->npts, s->nxyz, s->nmeta);
    }
    s->next = g_states;
    g_states = s;
    *out = s;
    return 0;
}

static int get_state(void *app, gpu_state **out)
{
    gpu_state *s = find_state(app);
    if (s) { *out = s; return 0; }
    return create_state((IGA *)app, 0, out);
}

PetscErrorCode snesiga_gpu_init(void *app_, int device)
{
    if (find_state(app_)) return 0;
    gpu_state *s;
    return create_state((IGA *)app_, device, &s);
}

PetscErrorCode snesiga_gpu_free(void *app_)
{
    gpu_state **pp = &g_states;
    while (*pp) {
        if ((*pp)->app == (IGA *)app_) {
            gpu_state *s = *pp;
            *pp = s->next;
            igab_destroy(s->ctx);
            free(s->nxyz); free(s->nmeta); free(s->nval); free(s->nwatch_copy); free(s->vals32);
            free(s);
            return 0;
        }
        pp = &(*pp)->next;
    }
    return 0;
}

int snesiga_gpu_set_neumann(void *app_, neumann_fn fn)
{
    gpu_state *s;
    int rc = get_state(app_, &s);
    if (rc) return rc;
    s->nfn = fn;
    s->neu_done = 0;
    return 0;
}

int snesiga_gpu_set_neumann_policy(void *app_, int policy, int n_watch)
{
    gpu_state *s;
    int rc = get_state(app_, &s);
    if (rc) return rc;
    if (policy < 0 || policy > 2 || (policy == 2 && n_watch < 1)) return PETSC_ERR_SUP;
    s->npol = policy;
    s->nwatch = n_watch;
    free(s->nwatch_copy);
    s->nwatch_copy = NULL;
    s->neu_done = 0;
    return 0;
}

int snesiga_gpu_set_tangent_precision(void *app_, int prec)
{
    gpu_state *s;
    int rc = get_state(app_, &s);
    if (rc) return rc;
    if (prec != IGAB_PREC_FP64 && prec != IGAB_PREC_FP32) return PETSC_ERR_SUP;
    s->prec = prec;
    return 0;
}

void *snesiga_gpu_context(void *app_)
{
    gpu_state *s = find_state(app_);
    return s ? (void *)s->ctx : NULL;
}

int snesiga_gpu_last_timings(void *app_, double ms[4])
{
    gpu_state *s = find_state(app_);
    if (!s) return PETSC_ERR_SUP;
    memcpy(ms, s->ms, sizeof(s->ms));
    return 0;
}

/* parameters the application may change between callbacks */
static int sync_params(gpu_state *s)
{
    IGA *app = s->app;
    int rc = igab_set_par_mat(s->ctx, app->phys->par_mat);
    if (!rc) rc = igab_set_par_dirichlet(s->ctx, app->bc->par_dirichlet);
    if (!rc) rc = igab_set_par_periodic(s->ctx, app->bc->par_periodic);
    if (!rc && app->phys->torder > 0)
        for (int lev = 1; lev <= app->phys->torder && !rc; lev++)
            rc = igab_set_history(s->ctx, lev, app->U_hist + (size_t)lev * (size_t)app->nselfIdx, 0);
    return rc;
}

/* evaluate the application's traction at the surface Gauss points
 * (the neumann() calls of src/snesiga_Residual.c:264 and :304) */
static int sync_neumann(gpu_state *s)
{
    if (s->npts == 0) return 0;
    double *pn = s->app->bc->par_neumann;
    if (s->neu_done) {
        if (s->npol == 1) return 0;
        if (s->npol == 2 && s->nwatch_copy && memcmp(s->nwatch_copy, pn, (size_t)s->nwatch * sizeof(double)) == 0) return 0;
    }
    if (!s->nfn) {
        fprintf(stderr, "snesiga_b200: Neumann boundaries present but no neumann() hook is defined\n");
        return IGAB_ERR_ARG;
    }
    for (long k = 0; k < s->npts; k++) {
        double xq[3] = {s->nxyz[3 * k], s->nxyz[3 * k + 1], s->nxyz[3 * k + 2]};
        double v = 0.0;
        s->nfn(&v, pn, s->nmeta[3 * k], s->nmeta[3 * k + 1], s->nmeta[3 * k + 2], xq);
        s->nval[k] = v;
    }
    if (s->npol == 2) {
        if (!s->nwatch_copy) s->nwatch_copy = (double *)malloc((size_t)s->nwatch * sizeof(double));
        if (s->nwatch_copy) memcpy(s->nwatch_copy, pn, (size_t)s->nwatch * sizeof(double));
    }
    s->neu_done = 1;
    return igab_set_neumann_values(s->ctx, s->nval);
}

static void keep_history(IGA *app, const PetscScalar *u)
{
    memcpy(app->U_hist, u, (size_t)app->nselfIdx * sizeof(double));
}

PetscErrorCode snesiga_b200_Residual(SNES snes, Vec U_, Vec Residual_, void *app_)
{
    (void)snes;
    double t0 = now_ms();
    gpu_state *s;
    int rc = get_state(app_, &s);
    if (rc) return rc;
    const PetscScalar *u;
    PetscScalar *r;
    VecGetArrayRead(U_, &u);
    keep_history(s->app, u);
    rc = sync_params(s);
    if (!rc) rc = sync_neumann(s);
    if (!rc) {
        VecGetArray(Residual_, &r);
        rc = igab_residual(s->ctx, u, r);
        VecRestoreArray(Residual_, &r);
    }
    VecRestoreArrayRead(U_, &u);
    VecAssemblyBegin(Residual_);
    VecAssemblyEnd(Residual_);
    s->ms[0] = now_ms() - t0;
    if (rc) fprintf(stderr, "snesiga_b200: residual failed: %s\n", igab_last_error());
    return map_err(rc);
}

/* Integrated densities of app->U_hist (level 0 is the iterate the callbacks saw last;
 * phys/getime also reads history levels 1 and 2) -- replaces src/iga_intdensity.c:10.
 * The reference has no error return: on failure every density is NaN and the
 * error is printed. */
void snesiga_b200_intdensity(double HH_[], void *app_)
{
    IGA *app = (IGA *)app_;
    const int nd = app && app->phys ? app->phys->ndensity : 0;
    gpu_state *s;
    int rc = get_state(app_, &s);
    if (!rc) rc = sync_params(s);
    if (!rc) rc = sync_neumann(s);
    if (!rc) {
        int n = 0;
        rc = igab_ndensity(s->ctx, &n);
        if (!rc && n != nd) {
            fprintf(stderr, "snesiga_b200: phys declares %d densities, the GPU path computes %d\n", nd, n);
            rc = IGAB_ERR_ARG;
        }
    }
    if (!rc) rc = igab_intdensity(s->ctx, app->U_hist, HH_);
    if (rc) {
        fprintf(stderr, "snesiga_b200: intdensity failed: %s\n", igab_last_error());
        for (int i = 0; i < nd; i++) HH_[i] = NAN;
    }
}

void iga_intdensity(double HH_[], void *app_) { snesiga_b200_intdensity(HH_, app_); }

/* Knot-insertion refinement of a solution -- replaces mesh/nurbs/nurbs_knotinsert.c:7
 * (same signature, ndim = 3, porder = 2); runs on GPU 0.  The reference asserts on a
 * bad argument: here the error is printed and the array is left unchanged. */
void nurbs_knotinsert(double *U_universal, const int nelem[], int nref, int porder, int ndim, int ndof,
                      int bc_periodic[])
{
    if (ndim != 3) {
        fprintf(stderr, "snesiga_b200: nurbs_knotinsert needs ndim = 3\n");
        return;
    }
    if (igab_knot_insert(U_universal, nelem, nref, porder, ndof, bc_periodic, 0))
        fprintf(stderr, "snesiga_b200: nurbs_knotinsert failed: %s\n", igab_last_error());
}

/* Solution files -- replace src/ioutil.c:89 and :126 on one rank: levels ihist0 ..
 * ihist1 - 1 of U_hist (iocomm->nDof values each) in universal order
 * (iocomm->universalIdx), raw doubles, level after level. */
void write_solution(const char *fname, double *U_hist, void *iocomm_, int ihist0, int ihist1)
{
    IOcomm *io = (IOcomm *)iocomm_;
    const long n = io->nDof, nl = ihist1 - ihist0;
    double *buf = (double *)malloc((size_t)(nl > 0 ? nl : 1) * (size_t)(io->nDof_global > 0 ? io->nDof_global : 1) * sizeof(double));
    if (!buf) {
        fprintf(stderr, "snesiga_b200: write_solution: out of memory\n");
        return;
    }
    for (long l = 0; l < nl; l++)
        for (long i = 0; i < n; i++) buf[l * io->nDof_global + io->universalIdx[i]] = U_hist[(ihist0 + l) * n + i];
    if (igab_write_solution(fname, buf, io->nDof_global, 0, (int)nl))
        fprintf(stderr, "snesiga_b200: write_solution failed: %s\n", igab_last_error());
    free(buf);
}

void read_solution(const char *fname, double *U_hist, void *iocomm_, int ihist0, int ihist1)
{
    IOcomm *io = (IOcomm *)iocomm_;
    const long n = io->nDof, nl = ihist1 - ihist0;
    double *buf = (double *)malloc((size_t)(nl > 0 ? nl : 1) * (size_t)(io->nDof_global > 0 ? io->nDof_global : 1) * sizeof(double));
    if (!buf) {
        fprintf(stderr, "snesiga_b200: read_solution: out of memory\n");
        return;
    }
    if (igab_read_solution(fname, buf, io->nDof_global, 0, (int)nl)) {
        fprintf(stderr, "snesiga_b200: read_solution failed: %s\n", igab_last_error());
    } else {
        for (long l = 0; l < nl; l++)
            for (long i = 0; i < n; i++) U_hist[(ihist0 + l) * n + i] = buf[l * io->nDof_global + io->universalIdx[i]];
    }
    free(buf);
}

/* Put the structured AIJ pattern into P the first time (as the reference's
 * first MatSetValues pass does) and check that P's CSR is exactly it. */
static int ensure_pattern(gpu_state *s, Mat P)
{
    if (s->pattern_ok == P) return 0;
    PetscBool assembled = PETSC_FALSE;
    MatAssembled(P, &assembled);
    long ndof = s->ndof, nnz = s->nnz;
    int *rowptr = (int *)malloc(((size_t)ndof + 1) * sizeof(int));
    int *cols = (int *)malloc((size_t)nnz * sizeof(int));
    if (!rowptr || !cols) { free(rowptr); free(cols); return IGAB_ERR_NOMEM; }
    int rc = igab_csr_pattern(s->ctx, rowptr, cols);
    if (rc) { free(rowptr); free(cols); return rc; }
    if (!assembled) {
        int maxc = 0;
        for (long r = 0; r < ndof; r++)
            if (rowptr[r + 1] - rowptr[r] > maxc) maxc = rowptr[r + 1] - rowptr[r];
        double *zeros = (double *)calloc((size_t)maxc, sizeof(double));
        if (!zeros) { free(rowptr); free(cols); return IGAB_ERR_NOMEM; }
        for (long r = 0; r < ndof; r++) {
            PetscInt row = (PetscInt)r;
            MatSetValues(P, 1, &row, rowptr[r + 1] - rowptr[r], cols + rowptr[r], zeros, INSERT_VALUES);
        }
        free(zeros);
        MatAssemblyBegin(P, MAT_FINAL_ASSEMBLY);
        MatAssemblyEnd(P, MAT_FINAL_ASSEMBLY);
    }
    PetscInt n;
    const PetscInt *ia, *ja;
    PetscBool done;
    MatGetRowIJ(P, 0, PETSC_FALSE, PETSC_FALSE, &n, &ia, &ja, &done);
    int same = done && n == ndof && ia[ndof] == nnz;
    if (same) same = memcmp(ia, rowptr, ((size_t)ndof + 1) * sizeof(int)) == 0 &&
                     memcmp(ja, cols, (size_t)nnz * sizeof(int)) == 0;
    MatRestoreRowIJ(P, 0, PETSC_FALSE, PETSC_FALSE, &n, &ia, &ja, &done);
    free(rowptr);
    free(cols);
    if (!same) {
        fprintf(stderr, "snesiga_b200: the tangent matrix does not have the structured AIJ pattern\n");
        return IGAB_ERR_ARG;
    }
    s->pattern_ok = P;
    return 0;
}

PetscErrorCode snesiga_b200_Tangent(SNES snes, Vec U_, Mat Tangent_, Mat Pmat_, void *app_)
{
    (void)snes;
    double t0 = now_ms();
    gpu_state *s;
    int rc = get_state(app_, &s);
    if (rc) return rc;
    const PetscScalar *u;
    VecGetArrayRead(U_, &u);
    keep_history(s->app, u);
    rc = sync_params(s);
    if (!rc) rc = ensure_pattern(s, Pmat_);
    if (!rc) {
        PetscScalar *a;
        MatSeqAIJGetArray(Pmat_, &a);
        if (s->prec == IGAB_PREC_FP64) {
            rc = igab_tangent(s->ctx, u, a, IGAB_PREC_FP64);
        } else {
            /* FP32 values land in the upper half of the double array (bytes 4*nnz..8*nnz);
             * widening in ascending order reads f[k] before any write reaches it */
            float *f = (float *)((char *)a + 4 * (size_t)s->nnz);
            rc = igab_tangent(s->ctx, u, f, IGAB_PREC_FP32);
            if (!rc)
                for (long k = 0; k < s->nnz; k++) a[k] = (double)f[k];
        }
        MatSeqAIJRestoreArray(Pmat_, &a);
    }
    VecRestoreArrayRead(U_, &u);
    if (!rc && Tangent_ != Pmat_) {
        MatAssemblyBegin(Tangent_, MAT_FINAL_ASSEMBLY);
        MatAssemblyEnd(Tangent_, MAT_FINAL_ASSEMBLY);
    }
    s->ms[1] = now_ms() - t0;
    if (rc) fprintf(stderr, "snesiga_b200: tangent failed: %s\n", igab_last_error());
    return map_err(rc);
}

PetscErrorCode snesiga_Residual(SNES snes, Vec U_, Vec Residual_, void *app_)
{
    return snesiga_b200_Residual(snes, U_, Residual_, app_);
}

PetscErrorCode snesiga_Tangent(SNES snes, Vec U_, Mat Tangent_, Mat Pmat_, void *app_)
{
    return snesiga_b200_Tangent(snes, U_, Tangent_, Pmat_, app_);
}

/* the points of halo block b (0-6 = z, y, x, yz, xz, xy, xyz) on the local grid of
 * nelem + p points per direction: along the block's directions the first p owned layers
 * (send) or the p ghost layers after the owned ones (recv), all owned points along the
 * others; dof indices in x, y, z, dof order (src/snesiga_init.c:186-330) */
static int halo_block(const int nb[3], const int nel[3], int p, int ndof, int b, int recv, int *out)
{
    static const int dims[7] = {1, 2, 4, 3, 5, 6, 7};   /* bit 2: x, bit 1: y, bit 0: z */
    int lo[3], hi[3];
    for (int d = 0; d < 3; d++) {
        const int in = (dims[b] >> (2 - d)) & 1;
        lo[d] = in && recv ? nb[d] : 0;
        hi[d] = in ? lo[d] + p : nb[d];
    }
    const int ny = nel[1] + p, nz = nel[2] + p;
    int n = 0;
    for (int x = lo[0]; x < hi[0]; x++)
        for (int y = lo[1]; y < hi[1]; y++)
            for (int z = lo[2]; z < hi[2]; z++)
                for (int k = 0; k < ndof; k++) {
                    if (out) out[n] = ndof * ((ny * nz) * x + nz * y + z) + k;
                    n++;
                }
    return n;
}

/* Single-rank snesiga_init (src/snesiga_init.c:12-132 with nproc = 1): the rank's
 * index maps (src/snesiga_init.c:134-330; along a periodic direction the halo
 * blocks are messages to itself, so a ghost's global index is its owner's), universal
 * = local ordering, one sequential AIJ matrix preallocated with the row lengths of
 * the owned pattern (src/snesiga_init.c:341-359 plus the wrapped neighbours of a
 * periodic direction), callbacks installed. */
void snesiga_init(void *app_, void *phys_, void *nurbs_, void *bc_, void *snesassmbl_, void *iocomm_)
{
    IGA *app = (IGA *)app_;
    Phys *phys = (Phys *)phys_;
    Nurbs *nurbs = (Nurbs *)nurbs_;
    SNESAssmbl *sa = (SNESAssmbl *)snesassmbl_;
    IOcomm *io = (IOcomm *)iocomm_;
    int ndof = phys->ndof, p = nurbs->porder;
    int *nb = nurbs->nbasis;
    app->phys = phys;
    app->nurbs = nurbs;
    app->bc = (BC *)bc_;
    int nproc = 1;
    MPI_Comm_size(MPI_COMM_WORLD, &nproc);
    int self_only = nproc == 1;
    for (int i = 0; i < nurbs->nsendPart; i++) self_only = self_only && nurbs->sendPart[i] == 0;
    for (int i = 0; i < nurbs->nrecvPart; i++) self_only = self_only && nurbs->recvPart[i] == 0;
    if (!self_only)
        fprintf(stderr, "snesiga_b200: snesiga_init supports one rank (periodic directions as its own halo); "
                        "callbacks will fail\n");
    int n = ndof * nb[0] * nb[1] * nb[2];
    app->nselfIdx = n;
    app->selfIdx = (int *)malloc((size_t)n * sizeof(int));
    {
        const int *nel = nurbs->nelem, ny = nel[1] + p, nz = nel[2] + p;
        int ia = 0;
        for (int x = 0; x < nb[0]; x++)
            for (int y = 0; y < nb[1]; y++)
                for (int z = 0; z < nb[2]; z++)
                    for (int k = 0; k < ndof; k++) app->selfIdx[ia++] = ndof * ((ny * nz) * x + nz * y + z) + k;
    }
    app->sendPtr = (int *)calloc((size_t)nurbs->nsendPart + 1, sizeof(int));
    app->recvPtr = (int *)calloc((size_t)nurbs->nrecvPart + 1, sizeof(int));
    for (int i = 0; i < nurbs->nsendPart; i++)
        app->sendPtr[i + 1] = app->sendPtr[i] + halo_block(nb, nurbs->nelem, p, ndof, nurbs->sendBlock[i], 0, NULL);
    for (int i = 0; i < nurbs->nrecvPart; i++)
        app->recvPtr[i + 1] = app->recvPtr[i] + halo_block(nb, nurbs->nelem, p, ndof, nurbs->recvBlock[i], 1, NULL);
    app->nsendIdx = app->sendPtr[nurbs->nsendPart];
    app->nrecvIdx = app->recvPtr[nurbs->nrecvPart];
    app->sendIdx = (int *)malloc((size_t)(app->nsendIdx > 0 ? app->nsendIdx : 1) * sizeof(int));
    app->recvIdx = (int *)malloc((size_t)(app->nrecvIdx > 0 ? app->nrecvIdx : 1) * sizeof(int));
    for (int i = 0; i < nurbs->nsendPart; i++)
        halo_block(nb, nurbs->nelem, p, ndof, nurbs->sendBlock[i], 0, app->sendIdx + app->sendPtr[i]);
    for (int i = 0; i < nurbs->nrecvPart; i++)
        halo_block(nb, nurbs->nelem, p, ndof, nurbs->recvBlock[i], 1, app->recvIdx + app->recvPtr[i]);
    io->nDof = n;
    io->nDof_array = (int *)malloc(sizeof(int));
    io->nDof_array[0] = n;
    io->iDof_displ_array = (int *)malloc(2 * sizeof(int));
    io->iDof_displ_array[0] = 0;
    io->iDof_displ_array[1] = n;
    io->nDof_global = n;
    io->universalIdx = (int *)malloc((size_t)n * sizeof(int));
    for (int c = 0, ia = 0; c < nb[0] * nb[1] * nb[2]; c++)
        for (int d = 0; d < ndof; d++) io->universalIdx[ia++] = ndof * nurbs->universalIdx_temp[c] + d;
    free(nurbs->universalIdx_temp);
    nurbs->universalIdx_temp = NULL;
    app->U_hist = (double *)malloc((size_t)(phys->torder + 1) * (size_t)n * sizeof(double));
    app->globalIdx = (int *)malloc((size_t)(n + app->nrecvIdx) * sizeof(int));
    for (int i = 0; i < n; i++) app->globalIdx[app->selfIdx[i]] = i;
    /* the blocks sent to itself come back in order: a ghost takes its owner's global index */
    if (self_only && app->nsendIdx == app->nrecvIdx)
        for (int i = 0; i < app->nrecvIdx; i++) app->globalIdx[app->recvIdx[i]] = app->globalIdx[app->sendIdx[i]];
    VecCreateMPI(MPI_COMM_WORLD, n, n, &sa->Residual_);
    VecDuplicate(sa->Residual_, &sa->U);
    int *d_nz = (int *)malloc((size_t)n * sizeof(int));
    int ia = 0;
    int per[3];
    for (int d = 0; d < 3; d++) per[d] = nb[d] == nurbs->nelem[d];   /* owned = elements: periodic */
    for (int x = 0; x < nb[0]; x++)
        for (int y = 0; y < nb[1]; y++)
            for (int z = 0; z < nb[2]; z++) {
                int cx = per[0] ? (nb[0] < 5 ? nb[0] : 5) : (x < p ? x : p) + 1 + (x > nb[0] - 1 - p ? nb[0] - 1 - x : p);
                int cy = per[1] ? (nb[1] < 5 ? nb[1] : 5) : (y < p ? y : p) + 1 + (y > nb[1] - 1 - p ? nb[1] - 1 - y : p);
                int cz = per[2] ? (nb[2] < 5 ? nb[2] : 5) : (z < p ? z : p) + 1 + (z > nb[2] - 1 - p ? nb[2] - 1 - z : p);
                for (int d = 0; d < ndof; d++) d_nz[ia++] = ndof * cx * cy * cz;
            }
    MatCreateAIJ(MPI_COMM_WORLD, n, n, n, n, 0, d_nz, 0, NULL, &sa->Tangent_);
    free(d_nz);
    free(nurbs->sendBlock);
    free(nurbs->recvBlock);
    nurbs->sendBlock = NULL;
    nurbs->recvBlock = NULL;
    MatSetOption(sa->Tangent_, MAT_KEEP_NONZERO_PATTERN, PETSC_TRUE);
    MatSetOption(sa->Tangent_, MAT_NO_OFF_PROC_ZERO_ROWS, PETSC_TRUE);
    MatSetOption(sa->Tangent_, MAT_SUBSET_OFF_PROC_ENTRIES, PETSC_TRUE);
    sa->snes_Residual = snesiga_b200_Residual;
    sa->snes_Tangent = snesiga_b200_Tangent;
    link_snesassmbl(snesassmbl_, app_);
}

int snesiga_gpu_set_ksp(void *app_, double rtol, int maxit)
{
    gpu_state *s;
    int rc = get_state(app_, &s);
    if (rc) return rc;
    if (rtol < 0.0 || maxit < 0) return PETSC_ERR_SUP;
    s->ksp_rtol = rtol;
    s->ksp_maxit = maxit;
    return 0;
}

int snesiga_gpu_last_solve(void *app_, igab_newton_info *info)
{
    gpu_state *s = find_state(app_);
    if (!s || !info) return PETSC_ERR_SUP;
    *info = s->last_solve;
    return 0;
}

static const char *reason_name(int r)
{
    switch (r) {
    case IGAB_SNES_DIVERGED_FNORM_NAN: return "DIVERGED_FNORM_NAN";
    case IGAB_SNES_DIVERGED_MAX_IT: return "DIVERGED_MAX_IT";
    case IGAB_SNES_DIVERGED_LINE_SEARCH: return "DIVERGED_LINE_SEARCH";
    default: return "DIVERGED";
    }
}

/* The reference application's solver loop on the GPU -- replaces src/snes_solve.c:10
 * (snes_solve), run with the SNES settings of src/snes_init.c:8-47.  The initial guess
 * is snesassmbl->U, the solution goes back there; app->U_hist[0..nselfIdx) holds it
 * afterwards and snesassmbl->Residual_ the residual at it, as after the reference's
 * loop.  Every residual, tangent and Krylov solve stays on the device
 * (igab_newton_solve): no tangent is copied to the host AIJ matrix.  Prints the
 * reference's line per subiteration; sets snesassmbl->converged. */
void snesiga_b200_solve(void *snesassmbl_)
{
    SNESAssmbl *sa = (SNESAssmbl *)snesassmbl_;
    void *app_ = app_of_snesassmbl(snesassmbl_);
    gpu_state *s = NULL;
    int rc = app_ ? get_state(app_, &s) : IGAB_ERR_ARG;
    if (!app_) fprintf(stderr, "snesiga_b200: snes_solve: this SNESAssmbl was not set up by snesiga_init\n");
    if (!rc) rc = sync_params(s);
    if (!rc) rc = sync_neumann(s);
    double *dU = NULL;
    if (!rc) rc = igab_device_buffers(s->ctx, &dU, NULL, NULL, IGAB_PREC_FP64);
    PetscScalar *u = NULL;
    if (!rc) {
        VecGetArray(sa->U, &u);
        rc = igab_upload(s->ctx, u, dU, s->ndof);
    }
    if (!rc) {
        igab_newton_opts o;
        igab_newton_defaults(&o);
        o.prec = s->prec;
        if (s->ksp_rtol > 0.0) o.ksp_rtol = s->ksp_rtol;
        if (s->ksp_maxit > 0) o.ksp_maxit = s->ksp_maxit;
        o.verbose = 1;
        memset(&s->last_solve, 0, sizeof(s->last_solve));
        rc = igab_newton_solve(s->ctx, dU, &o, &s->last_solve, NULL, NULL, 0);
    }
    if (!rc) rc = igab_download(s->ctx, dU, u, s->ndof);
    if (u) {
        if (!rc) keep_history(s->app, u);
        VecRestoreArray(sa->U, &u);
    }
    if (!rc) {
        /* the residual at the solution in Residual_, as SNES leaves its function vector */
        const PetscScalar *uc;
        PetscScalar *r;
        VecGetArrayRead(sa->U, &uc);
        VecGetArray(sa->Residual_, &r);
        rc = igab_residual(s->ctx, uc, r);
        VecRestoreArray(sa->Residual_, &r);
        VecRestoreArrayRead(sa->U, &uc);
    }
    if (rc) {
        fprintf(stderr, "snesiga_b200: snes_solve failed: %s\n", igab_last_error());
        sa->converged = 0;
        return;
    }
    if (!s->last_solve.converged) printf("%s.\n", reason_name(s->last_solve.reason));
    sa->converged = s->last_solve.converged ? 1 : 0;
}

void snes_solve(void *snesassmbl_) { snesiga_b200_solve(snesassmbl_); }
