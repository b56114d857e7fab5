/*
 * Internal state of an assembly context (not part of the ABI).
 */
#ifndef IGAB_INTERNAL_H
#define IGAB_INTERNAL_H

#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include <vector>
#include "igab.h"
#include "igab_math.cuh"

#define IGAB_NQ 4         /* Gauss points per direction (src/snesiga_Residual.c:99) */
#define IGAB_NQ3 64
#define IGAB_TAB1D 36     /* doubles per element per direction: [q 4][l 3][k 3] */

/* Everything a kernel needs about the mesh and physics, passed by value. */
struct igab_geom {
    int ne[3];            /* elements per direction */
    int nb[3];            /* control points per direction = ne + 2 */
    long ndof;
    const double *tab[3]; /* 1-D basis tables [e][q][l][k] */
    const double *wh[3];  /* [e][q] Gauss weight times element length */
    const double *xq[3];  /* [e][q] Gauss point coordinate */
    const int *rowptr;    /* CSR row pointer [ndof+1] */
    igab_ge_coef coef;
    double pp[9];         /* par_periodic */
    int periodic;         /* any pp != 0 */
    /* transient (phys/getime): history pointers and time-integration scalars */
    const double *hist1;  /* U at t_n     (U_hist level 1) */
    const double *hist0;  /* U at t_{n-1} (U_hist level 2) */
    double rho, cii, dt;
    int phys;
    /* per-element integrand scale s_e = exp(g_e), element e = (ex*ne1 + ey)*ne2 + ez; null: 1 */
    const double *escale;
    /* phys/getime tangent-type assembly: weights w_j of the Hessian Taylor coefficients H_j
     * (j = 0..3) and the coefficient of the value-component mass term; the tangent d r/d u
     * is w = (1/4, 1/6, 1/8, 0), mass rho/dt^2 + c/(2 dt) (igab_getime.cu) */
    double tw[4];
    double tmass;
};

/* Batched assembly: the work list of a persistent launch over many meshes.
 * item = (instance, sweep position p, tile, colour), ordered colour-major in the
 * batch's colour order (colour = igab_colour_at(order, p)); done[8 i + p] counts the
 * finished tiles of position p of instance i, need[8 i + p] how many there are.  A
 * tile of position p starts once every earlier position of its instance is complete
 * (bounded wait), so tiles of one instance never overlap in time unless they are of
 * one colour. */
struct igab_batch_dev {
    const igab_geom *geoms;
    const int4 *items;
    int nitems;
    int *counter;          /* next item; zeroed before each launch (with done) */
    int *done;
    const int *need;
    const long *dof_off;   /* [n] offsets of the instances in U / R */
    const long *nnz_off;   /* [n] offsets in the CSR values */
    int *status;           /* bit 1: a dependency wait gave up */
    long spin_limit;       /* polls before a dependency wait gives up */
    int hold;              /* added to need[0] of instance 0 (test switch; 0 in normal use) */
};

#define IGAB_MAX_SLABS 32   /* x-slabs of the host-pointer tangent */

struct igab_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;

    int phys = IGAB_PHYS_GE;
    int torder = 0;
    int ne[3] = {0, 0, 0}, nb[3] = {0, 0, 0};
    long ncp = 0, ndof = 0, nnz = 0, nel = 0;
    std::vector<double> knots[3];
    double par_mat[9], par_dirichlet[9], par_periodic[9];
    int bc_type[36];

    /* host copies */
    std::vector<int> rowptr_h;
    double gauss_x[IGAB_NQ], gauss_w[IGAB_NQ];

    /* device: tables */
    double *d_tab[3] = {nullptr, nullptr, nullptr};
    double *d_wh[3] = {nullptr, nullptr, nullptr};
    double *d_xq[3] = {nullptr, nullptr, nullptr};
    int *d_rowptr = nullptr;

    /* Dirichlet: unique rows, last-written value (residual) */
    long nd = 0;
    int *d_drow = nullptr;
    double *d_dg = nullptr;
    bool dirichlet_dirty = true;

    /* Neumann: active (face, order, dof) combos in the reference's loop order */
    struct combo { int face, order, dof; long offset; int ne0, ne1; };
    std::vector<combo> combos;
    long n_neu_points = 0;
    double *d_hval = nullptr;          /* traction values at surface Gauss points */
    bool neumann_nonzero = false;
    long n_neu_rows = 0;               /* rows receiving Neumann terms */
    int *d_neu_row = nullptr;          /* dof per row */
    int *d_neu_ptr = nullptr;          /* [n_neu_rows+1] into entries */
    int4 *d_neu_ent = nullptr;         /* (combo, layer slot, bx, by) */
    double *d_dnz = nullptr;           /* [6 faces][2 layers] normal derivative of the basis at the face */
    int *d_combo_info = nullptr;       /* [ncombo][8]: face, order, dof, ne0, ne1, offset_lo, offset_hi, dir map */

    /* history (transient) */
    double *d_hist = nullptr;          /* [torder][ndof] */

    /* owned scratch for the host-pointer entry points */
    double *d_U = nullptr, *d_R = nullptr;
    void *d_vals = nullptr;
    int vals_prec = -1;

    int tile_res = 2, tile_tan = 2;
    int tan_kernel = 1;   /* FP64 tangent: 1 tensor-core (mma f64), 0 SIMT */
    int tan32_kernel = 1; /* FP32 tangent: 1 tcgen05 tensor cores (TF32 hi/lo), 0 SIMT */
    int colour_order = 0; /* igab_colour_order */
    int *d_status = nullptr;   /* device status word: nonzero after a bounded wait gave up */
    int last_launches = 0;

    /* profiling events: [0..2] residual (start, after volume, end), [3..5] tangent */
    bool profiling = false;
    cudaEvent_t ev[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    bool ev_res = false, ev_tan = false;
    int nvol_res = 0, nvol_tan = 0;

    /* adjoint: element scales and the masked adjoint vector */
    double *d_escale = nullptr;        /* [nel] exp(g_e) */
    bool escale_on = false;
    double *d_lam = nullptr;           /* [ndof] lambda with Dirichlet rows zeroed */

    /* integrated densities: per-block partial rows, result */
    double *d_dens_part = nullptr;
    size_t dens_part_bytes = 0;
    double *d_HH = nullptr;

    /* host-pointer tangent: download stream, and one event per x-slab whose rows are final */
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t slab_ev[IGAB_MAX_SLABS] = {};

    /* device Newton solve (igab_newton.cu): F, G, Y, J Y, W and reduction scratch; tangent values */
    double *d_nl = nullptr;
    double *h_nl = nullptr;            /* pinned, 2 doubles */
    void *d_nl_vals = nullptr;
    size_t nl_vals_bytes = 0;

    /* multigrid hierarchy of the Krylov solve (igab_mg.cu), rebuilt when param_version changes */
    struct igab_mg *mg = nullptr;
    long param_version = 0;            /* bumped by every change of par_mat, par_periodic, element scales */

    /* assembly graphs of the device Newton solve (igab_newton.cu), re-captured when
     * sched_version changes */
    struct igab_nl_graphs *nlg = nullptr;
    long sched_version = 0;            /* bumped by every change of a kernel parameter (par_mat, par_periodic,
                                          Dirichlet rows, element scales) or of the schedule (tiles, kernels) */

    /* periodic directions: the kernels run on the local grid (nb), the owned system
     * (igab_periodic.cu) gathers, folds and applies the Dirichlet rows */
    int periodic[3] = {0, 0, 0};
    struct igab_periodic *per = nullptr;

    /* captured assembly graph */
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    bool force_neumann = false;   /* graph capture keeps the Neumann kernel in whatever the values become */

    igab_geom geom() const;
};

/* the k-th colour swept under colour order `order` (igab_colour_order); every order sweeps
 * the even-x colours (0-3) first */
__host__ __device__ inline int igab_colour_at(int order, int k)
{
    if (order == 1) return (k & 4) | (3 - (k & 3));   /* 3,2,1,0,7,6,5,4 */
    if (order == 2) return k ^ (k >> 1);              /* 0,1,3,2,6,7,5,4 */
    return k;
}

/* kernels / launchers (igab_kernels.cu) */
int igab_launch_residual(igab_ctx *c, const double *dU, double *dR);
int igab_launch_density(igab_ctx *c, const double *dU, double *dHH);   /* igab_density.cu */
/* igab_krylov.cu: K x on the structured pattern, Jacobi-BiCGStab on the device */
int igab_launch_spmv(igab_ctx *c, const void *dvals, int prec, const double *dx, double *dy);
int igab_krylov_solve(igab_ctx *c, const void *dvals, int prec, const double *db, double *dx, double rtol,
                      double atol, int maxit, int *iterations, int *converged, double *rnorm, double *bnorm);
void igab_krylov_release(igab_ctx *c);
void igab_newton_release(igab_ctx *c);   /* igab_newton.cu */
int igab_check_status(igab_ctx *c);      /* after a synchronisation: a bounded wait that gave up -> error */
/* entry points without a periodic form return IGAB_ERR_UNSUPPORTED for such a mesh */
#define IGAB_NO_PERIODIC(ctx, name)                                                                   \
    do {                                                                                              \
        if ((ctx) && (ctx)->per) {                                                                    \
            igab_set_error("%s: not available for a mesh with periodic directions", name);           \
            return IGAB_ERR_UNSUPPORTED;                                                              \
        }                                                                                             \
    } while (0)
/* igab_periodic.cu: the owned system of a mesh with periodic directions */
int igab_periodic_build(igab_ctx *c);
int igab_periodic_set_dirichlet(igab_ctx *c, const std::vector<int> &rows, const std::vector<double> &g);
int igab_periodic_residual(igab_ctx *c, const double *U_own, double *R_own);
int igab_periodic_tangent(igab_ctx *c, const double *U_own, void *V_own, int prec);
int igab_periodic_gather(igab_ctx *c, const double *U_own, double *U_loc);
int igab_periodic_dirichlet_rows(igab_ctx *c, long *n, int *rows);
void igab_periodic_release(igab_ctx *c);
long igab_periodic_ndof(const igab_ctx *c);
long igab_periodic_nnz(const igab_ctx *c);
const std::vector<int> &igab_periodic_rowptr(const igab_ctx *c);
const std::vector<int> &igab_periodic_cols(const igab_ctx *c);
/* igab_mg.cu: multigrid-preconditioned CG (breakdown: p.Kp <= 0) or GMRES on the context's tangent */
int igab_mg_solve(igab_ctx *c, int method, const void *vals, int prec, const double *b, double *x, double rtol,
                  double atol, int maxit, int *iterations, int *converged, double *rnorm, double *bnorm, int *breakdown);
int igab_mg_levels(igab_ctx *c, int *levels);
void igab_mg_release(igab_ctx *c);
int igab_launch_tangent(igab_ctx *c, const double *dU, void *dvals, int prec);
/* the same, slab by slab along x: after slab i, rows [0, row_end[i]) are final and
 * c->slab_ev[i] is recorded on c->stream (one slab when the kernels have no x-range) */
int igab_launch_tangent_slabs(igab_ctx *c, const double *dU, void *dvals, int prec, long *row_end, int *nslab);
int igab_launch_csr_cols(igab_ctx *c, int *dcols);
int igab_launch_check_finite(igab_ctx *c, const void *dev, long n, int prec, int *all_finite);
int igab_launch_basis_tables(igab_ctx *c, int d, const double *dkv, const double *dgx, const double *dgw);
int igab_launch_fma_peak(int prec, double *tflops);
int igab_launch_dmma_peak(double *tflops);   /* igab_tangent_dmma.cu */
/* tangent volume kernels over the tiles with x tile coordinate in [tx0, tx1) (tiles of 2 elements) */
int igab_launch_tan_dmma(igab_ctx *c, const double *dU, double *dv, int tx0, int tx1);
int igab_launch_tan_tc32(igab_ctx *c, const double *dU, float *dv, int tx0, int tx1);
/* persistent batched launches (igab_batch.cu builds the work list) */
int igab_launch_res_batch(const igab_batch_dev &B, int grid, cudaStream_t s, const double *dU, double *dR);
int igab_launch_tan_dmma_batch(const igab_batch_dev &B, int grid, cudaStream_t s, const double *dU, double *dv);
int igab_launch_tan_tc32_batch(const igab_batch_dev &B, int grid, cudaStream_t s, const double *dU, float *dv);
int igab_launch_tan_dirichlet_batch(const igab_batch_dev &B, long nd, const int *dinst, const int *drow, void *dv,
                                    int prec, cudaStream_t s);
/* R = U - g on a list of (global) Dirichlet rows */
int igab_launch_res_dirichlet_rows(long nd, const int *drow, const double *dg, const double *dU, double *dR,
                                   cudaStream_t s);
/* CTAs per SM the persistent kernels can hold (occupancy; the FP32 tangent is capped at 2 by its tensor memory) */
int igab_batch_occupancy_res(int *per_sm);
int igab_batch_occupancy_dmma(int *per_sm);
int igab_batch_occupancy_tc32(int *per_sm);
int igab_launch_tan_getime(igab_ctx *c, const double *dU, void *dv, int prec);
/* zero the Dirichlet rows of CSR values (rows only) */
int igab_launch_zero_csr_rows(igab_ctx *c, void *dv, int prec);
/* the same kernel with explicit weights (history Jacobians); level 0 = tangent */
int igab_launch_tan_getime_level(igab_ctx *c, const double *dU, void *dv, int prec, int level);
int igab_launch_exp_scale(igab_ctx *c, const double *dg);
int igab_launch_adjoint_dRdg(igab_ctx *c, const double *dU, const double *dlam, double *dgrad);
int igab_launch_tangent_transpose(igab_ctx *c, const void *dvals, int prec, const double *dx, double *dy);
/* record profiling event k on the context stream if profiling is on */
static inline void igab_mark(igab_ctx *c, int k)
{
    if (c->profiling && c->ev[k]) cudaEventRecord(c->ev[k], c->stream);
}

/* error helpers (igab_capi.cu) */
void igab_set_error(const char *fmt, ...);
#define IGAB_CUDA_TRY(call)                                                        \
    do {                                                                           \
        cudaError_t _e = (call);                                                   \
        if (_e != cudaSuccess) {                                                   \
            igab_set_error("%s:%d %s: %s", __FILE__, __LINE__, #call,             \
                           cudaGetErrorString(_e));                                \
            return IGAB_ERR_CUDA;                                                  \
        }                                                                          \
    } while (0)

#endif
