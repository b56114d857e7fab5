/*
 * igab.h -- plain C ABI of the B200 element-assembly library (libigap4_b200.so).
 *
 * One context = one single-rank IGA mesh (quadratic C1 B-splines, p = 2,
 * 4x4x4 Gauss points per element) plus its physics, boundary tables and
 * device buffers.  Entry points take plain pointers and sizes; every one
 * returns 0 on success or a nonzero igab_status.  Nothing here needs PETSc.
 *
 * The reference interface each entry point replaces (IGAP4STANDARD paths):
 *   igab_create              snesiga_init            src/snesiga_init.c:12-132
 *                            (index maps, AIJ preallocation; single rank)
 *   igab_csr_pattern         MatCreateAIJ + first MatSetValues pattern
 *                            src/snesiga_init.c:115-124, :341-359
 *   igab_residual[_device]   snesiga_Residual        src/snesiga_Residual.c:13-417
 *   igab_tangent[_device]    snesiga_Tangent         src/snesiga_Tangent.c:13-284
 *   igab_set_history         app->U_hist levels 1..torder   include/iga.h:14
 *   igab_neumann_points /    the neumann() hook evaluated at the surface
 *   igab_set_neumann_values  Gauss points            src/snesiga_Residual.c:243-320
 *   igab_set_par_*           Phys.par_mat, BC.par_dirichlet/par_periodic
 *                            include/phys.h:16, include/bc.h:6-8
 *
 * Numbering: dof = 3*(nb1*nb2*ix + nb2*iy + iz) + d with nb = nelem + 2
 * (src/snesiga_init.c:89-94, one rank).  The tangent is a CSR matrix with
 * ascending column indices per row and the exact AIJ pattern the reference
 * creates (every pair of control points whose supports overlap, 3x3 dofs).
 */
#ifndef IGAB_H
#define IGAB_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct igab_ctx igab_ctx;

enum igab_status {
    IGAB_OK = 0,
    IGAB_ERR_ARG = 1,        /* bad argument (size, pointer, enum) */
    IGAB_ERR_CUDA = 2,       /* a CUDA call failed; message in igab_last_error() */
    IGAB_ERR_NOMEM = 3,      /* host or device allocation failed */
    IGAB_ERR_NONFINITE = 4,  /* residual or tangent contains NaN/Inf */
    IGAB_ERR_UNSUPPORTED = 5 /* physics / order / precision not built */
};

enum igab_phys { IGAB_PHYS_GE = 0, IGAB_PHYS_GETIME = 1 };
enum igab_prec { IGAB_PREC_FP64 = 0, IGAB_PREC_FP32 = 1 };

typedef struct {
    int phys;                 /* igab_phys */
    int nelem[3];             /* elements per direction */
    const double *knots;      /* 3 knot vectors back to back, nelem[d]+5 values each (open, or the
                                 uniform extension of mesh/nurbs/nurbs_genuniform.c:40-43 along a
                                 periodic direction) */
    double par_mat[9];        /* {r, curv, e0, e345, le, rho, cii, dt, t} (phys/ge/init.c:17-18) */
    int bc_type[36];          /* [face][order][dof], 0 Dirichlet, 1 Neumann (include/bc.h:6) */
    double par_periodic[9];   /* affine F0 added at Gauss points (src/snesiga_Residual.c:140-144) */
    double par_dirichlet[9];  /* affine map of the Dirichlet values (src/iga_dirichlet.c:10-12) */
    int bc_periodic[3];       /* 1: the direction is periodic (nelem[d] >= 3 control points owned, no
                                 boundary faces; mesh/nurbs/nurbs_init.c:24-39 on one rank) */
} igab_mesh_desc;

/* Periodic directions (one rank).  The mesh owns nelem[d] control points along a periodic
 * direction (nelem[d] + 2 otherwise); dofs, the residual, the AIJ pattern (rows and columns
 * of every pair of owned points that share an element, ascending) and the tangent values
 * are in that owned numbering.  The kernels assemble on the local grid of nelem[d] + 2
 * points per direction, whose last two along a periodic direction are the ghosts of owned
 * points 0 and 1 (the halo the reference exchanges with itself, src/snesiga_Residual.c:54-74);
 * the ghost rows and columns are then added into their owners in a fixed order, and the
 * Dirichlet rows of the non-periodic faces applied on the owned system.  A periodic mesh
 * takes igab_residual[_device], igab_tangent[_device], igab_set_history, the pattern and
 * parameter calls; the other entry points return IGAB_ERR_UNSUPPORTED for it. */

/* ---- lifetime */
int igab_create(const igab_mesh_desc *desc, int device, igab_ctx **out);
int igab_destroy(igab_ctx *ctx);
const char *igab_last_error(void);
int igab_version(void);

/* ---- sizes and pattern */
int igab_sizes(const igab_ctx *ctx, long *ndof, long *nnz, long *nelem_total);
/* rowptr[ndof+1], cols[nnz] (host arrays; either may be NULL) */
int igab_csr_pattern(igab_ctx *ctx, int *rowptr, int *cols);
/* position of entry (row, col) in the CSR value array, or -1 if not in the pattern */
long igab_csr_offset(const igab_ctx *ctx, long row, long col);

/* ---- parameters (take effect at the next assembly) */
int igab_set_par_mat(igab_ctx *ctx, const double par_mat[9]);
int igab_set_par_dirichlet(igab_ctx *ctx, const double par_dirichlet[9]);
int igab_set_par_periodic(igab_ctx *ctx, const double par_periodic[9]);
/* the Dirichlet rows (dofs whose residual row is U - g, src/iga_dirichlet.c), ascending:
 * n receives the count, rows (NULL or n ints) the dofs */
int igab_dirichlet_rows(igab_ctx *ctx, long *n, int *rows);

/* ---- Neumann data: the caller evaluates its traction at the surface Gauss
 * points and hands the values over.  n_points = total point count; xyz
 * receives 3 coordinates per point, meta 3 ints per point (face, order, dof),
 * in the order the values must be given.  All-zero values skip the kernel. */
int igab_neumann_points(const igab_ctx *ctx, long *n_points, double *xyz, int *meta);
int igab_set_neumann_values(igab_ctx *ctx, const double *values);

/* ---- history levels 1..torder of U (transient physics): host or device pointer */
int igab_set_history(igab_ctx *ctx, int level, const double *U, int on_device);

/* ---- assembly.  _device variants take device pointers and enqueue on the
 * context stream; the host variants copy U in and the result out. */
int igab_residual(igab_ctx *ctx, const double *U_host, double *R_host);
int igab_residual_device(igab_ctx *ctx, const double *U_dev, double *R_dev);
/* vals: nnz doubles (IGAB_PREC_FP64) or floats (IGAB_PREC_FP32).  igab_tangent
 * assembles meshes of 23 or more elements along x slab by slab along x and downloads
 * the rows each slab finishes on a second stream while the next slabs are assembled
 * (pinned vals_host overlaps fully); the values are bitwise those of igab_tangent_device. */
int igab_tangent(igab_ctx *ctx, const double *U_host, void *vals_host, int prec);
int igab_tangent_device(igab_ctx *ctx, const double *U_dev, void *vals_dev, int prec);

/* ---- stream / sync / device scratch */
int igab_set_stream(igab_ctx *ctx, void *cuda_stream);
int igab_sync(igab_ctx *ctx);
/* device buffers owned by the context, sized ndof / nnz, for callers without an allocator */
int igab_device_buffers(igab_ctx *ctx, double **U_dev, double **R_dev, void **vals_dev, int prec);
/* n doubles host -> device / device -> host on the context's stream, synchronously
 * (for C callers that do not link the CUDA runtime; no reference counterpart) */
int igab_upload(igab_ctx *ctx, const double *host, double *dev, long n);
int igab_download(igab_ctx *ctx, const double *dev, double *host, long n);
/* check a device vector for NaN/Inf (1 = all finite) */
int igab_check_finite(igab_ctx *ctx, const void *dev, long n, int prec, int *all_finite);

/* ---- tuning: elements per tile edge of the 8-colour schedule (2 or 4), 0 = auto */
int igab_set_tile(igab_ctx *ctx, int residual_tile, int tangent_tile);
/* kernel choices: IGAB_OPT_TANGENT_FP64_KERNEL 1 = FP64 tensor path (mma f64), 0 = FP64 FMA pipe;
 * IGAB_OPT_TANGENT_FP32_KERNEL 1 = tcgen05 tensor cores (TF32 hi/lo split, FP32 accumulation in
 * tensor memory), 0 = FP32 FMA pipe.  IGAB_OPT_COLOUR_ORDER: the order in which the 8 colours
 * of the element schedule are swept (colour = 4 x-parity + 2 y-parity + z-parity):
 * IGAB_COLOURS_NATURAL 0..7, IGAB_COLOURS_MIRRORED 3,2,1,0,7,6,5,4, IGAB_COLOURS_GRAY
 * 0,1,3,2,6,7,5,4.  Each order fixes the order in which every CSR entry receives its
 * additions (results are bitwise repeatable per order; orders differ by rounding); all three
 * sweep the even-x colours first, which keeps the x-slab tangent of the host entry points
 * equal to the whole-mesh one. */
enum igab_option { IGAB_OPT_TANGENT_FP64_KERNEL = 1, IGAB_OPT_TANGENT_FP32_KERNEL = 2, IGAB_OPT_COLOUR_ORDER = 3 };
enum igab_colour_order { IGAB_COLOURS_NATURAL = 0, IGAB_COLOURS_MIRRORED = 1, IGAB_COLOURS_GRAY = 2 };
int igab_set_option(igab_ctx *ctx, int option, int value);
int igab_get_option(const igab_ctx *ctx, int option, int *value);
/* launches issued by the last assembly call (kernel count) */
int igab_last_launch_count(const igab_ctx *ctx, int *n);

/* ---- measurement: with profiling on, assembly calls record CUDA events on
 * the context stream around their kernel phases; igab_last_kernel_ms waits
 * for the stream and returns milliseconds of the last calls:
 * ms[0] residual volume kernels, ms[1] residual boundary kernels,
 * ms[2] tangent volume kernels, ms[3] tangent Dirichlet row/column zeroing,
 * ms[4] number of residual volume launches, ms[5] number of tangent volume launches */
int igab_set_profiling(igab_ctx *ctx, int on);
int igab_last_kernel_ms(igab_ctx *ctx, double ms[6]);
/* FMA throughput probe of the device (TFLOP/s, 2 flops per FMA), prec = igab_prec */
int igab_fma_peak(int device, int prec, double *tflops);
/* FP64 tensor-pipe throughput probe (TFLOP/s): back-to-back mma.sync m8n8k4 f64 on
 * independent accumulators, 32 warps per SM (the pipe of the FP64 tangent's products) */
int igab_dmma_peak(int device, double *tflops);
/* Check of the tcgen05 operand layout and descriptors used by the FP32 tensor-core tangent
 * (no reference counterpart): one CTA computes A B^T for fixed small-integer A (128 x 32) and
 * B (96 x 32) with the M 128 / N 96 and M 128 / N 32 instruction shapes; out (128 x 160 floats,
 * row-major) receives accumulator columns 0-95 (A B^T), 96-127 (A B[0:32]^T) and 128-159
 * (A B[0:32]^T over K 0-15 minus it over K 16-31, the negate-A form). */
int igab_tc_selftest(int device, float *out);
/* TF32 tensor-core throughput probe (TFLOP/s, dense): one CTA per SM issuing back-to-back
 * tcgen05.mma kind::tf32 M 128 x N n_cols x K 8 (n_cols 32, 96 = the FP32 tangent's
 * shapes, or 256 = full width); no reference counterpart. */
int igab_tc_peak(int device, int n_cols, double *tflops);

/* ---- CUDA graphs: capture one assembly at fixed device pointers, replay it.
 * what: 1 residual, 2 tangent, 3 both (residual then tangent).  Parameters
 * changed later with igab_set_par_dirichlet / igab_set_neumann_values /
 * igab_set_history are picked up by replays (they update device buffers in
 * place); igab_set_par_mat and igab_set_par_periodic need a new capture. */
int igab_graph_capture(igab_ctx *ctx, const double *U_dev, double *R_dev, void *vals_dev, int prec, int what);
int igab_graph_launch(igab_ctx *ctx);
int igab_graph_destroy(igab_ctx *ctx);

/* ---- discrete adjoint of the element-scaled problem (no reference counterpart).
 * Every element integrand (volume residual and tangent) is multiplied by
 * s_e = exp(g_e); element e = (ex*ne1 + ey)*ne2 + ez, the reference's element
 * loop order (src/snesiga_Residual.c:104-106).  Neumann and Dirichlet rows are
 * not scaled.
 *   forward : s = exp(g) (g_dev NULL keeps the current scales), then R and/or
 *             the CSR tangent at U, as igab_residual_device / igab_tangent_device.
 *   backward: KTlam = K^T lam on CSR values vals_dev (structured pattern) and/or
 *             grad[e] = sum_r lam_r dR_r/dg_e = s_e lam_e . R_e(U), Dirichlet rows
 *             of lam ignored (there R = U - g does not depend on g).
 * With K^T lam = dJ/dU solved by the caller, dJ/dg = -grad. */
int igab_set_element_log_scale(igab_ctx *ctx, const double *g, int on_device);   /* g NULL: s = 1 */
int igab_adjoint_forward(igab_ctx *ctx, const double *g_dev, const double *U_dev, double *R_dev,
                         void *vals_dev, int prec);
int igab_adjoint_backward(igab_ctx *ctx, const double *U_dev, const void *vals_dev, int prec,
                          const double *lam_dev, double *KTlam_dev, double *grad_dev);

/* ---- autotuner (no reference counterpart): times every candidate schedule on this
 * mesh and state (U_dev; NULL = zero state) with CUDA events on the context stream,
 * reps timed runs after one warm-up, and leaves the fastest applied.  what: bit 0
 * residual (elements per block: tile edge 2 or 4), bit 1 FP64 tangent (tensor path or FMA
 * pipe), bit 2 FP32 tangent (tcgen05 or FMA pipe), bit 3 colour order (the three orders of
 * IGAB_OPT_COLOUR_ORDER, timed on the sum of the kernels bits 0-2 select, all three when
 * none).  Times of the chosen candidates in ms. */
typedef struct {
    int residual_tile, tangent_fp64_kernel, tangent_fp32_kernel;
    double residual_ms, tangent_fp64_ms, tangent_fp32_ms;
    int colour_order;
} igab_tune_result;
int igab_autotune(igab_ctx *ctx, const double *U_dev, int what, int reps, igab_tune_result *out);

/* ---- batched assembly: many independent meshes of uneven size, each with its own
 * material constants and boundary tables, assembled by one persistent launch per
 * operator (no reference counterpart: the reference runs one mesh per process; each
 * instance's result is the single-mesh result of igab_residual_device /
 * igab_tangent_device bit for bit).  phys/ge only; Neumann tractions are zero.
 * Instance i owns U/R[dof_offsets[i] .. dof_offsets[i+1]) and
 * vals[nnz_offsets[i] .. nnz_offsets[i+1]) in its own numbering and AIJ pattern;
 * igab_batch_instance returns its context for pattern queries and parameter
 * changes (then call igab_batch_refresh).  Schedule knobs (the autotuner's search
 * space): CTAs per SM of the residual / FP64 tangent / FP32 tangent persistent
 * kernels (0 = as many as fit) and the instance order of the colour-major work
 * list (0 natural, 1 largest first). */
typedef struct igab_batch igab_batch;
int igab_batch_create(const igab_mesh_desc *descs, int n, int device, igab_batch **out);
int igab_batch_destroy(igab_batch *b);
int igab_batch_sizes(const igab_batch *b, long *ndof, long *nnz, long *nelem, long *dof_offsets, long *nnz_offsets);
igab_ctx *igab_batch_instance(igab_batch *b, int i);
int igab_batch_refresh(igab_batch *b);
int igab_batch_set_stream(igab_batch *b, void *cuda_stream);
int igab_batch_set_schedule(igab_batch *b, int ctas_res, int ctas_tan64, int ctas_tan32, int order);
int igab_batch_get_schedule(const igab_batch *b, int *ctas_res, int *ctas_tan64, int *ctas_tan32, int *order);
/* colour order of the batch's work list (igab_colour_order; natural by default) */
int igab_batch_set_colour_order(igab_batch *b, int colour_order);
int igab_batch_get_colour_order(const igab_batch *b, int *colour_order);
/* The launches below return once enqueued.  A tile of colour c waits (bounded) for the
 * earlier colours of its instance; a wait that gives up sets a status word and the
 * launch still ends, with that instance's R or values incomplete.  igab_batch_sync
 * (after igab_batch_residual_device, igab_batch_tangent_device or
 * igab_batch_graph_launch) reports it as IGAB_ERR_CUDA and clears it: check its
 * return before using the results. */
int igab_batch_residual_device(igab_batch *b, const double *U_dev, double *R_dev);
int igab_batch_tangent_device(igab_batch *b, const double *U_dev, void *vals_dev, int prec);
int igab_batch_sync(igab_batch *b);
/* colour-dependency wait: polls (128 ns apart) before a wait gives up, 0 = the default
 * 4,194,304; unreachable = 1 makes every wait on colour 0 of instance 0 run out (a test
 * switch for the give-up path; results are then incomplete).  No reference counterpart. */
int igab_batch_set_wait_limit(igab_batch *b, long polls, int unreachable);
int igab_batch_last_launch_count(const igab_batch *b, int *n);
/* one Newton iteration's assembly (residual then tangent) captured in a CUDA graph */
int igab_batch_graph_capture(igab_batch *b, const double *U_dev, double *R_dev, void *vals_dev, int prec);
int igab_batch_graph_launch(igab_batch *b);
/* autotuner of the batch schedule: CTAs per SM of each persistent kernel and the
 * instance order (what: bit 0 residual, bit 1 FP64 tangent, bit 2 FP32 tangent), and with
 * bit 3 the colour order (on the sum of the selected kernels, all three when none);
 * the fastest schedule is left applied. */
typedef struct {
    int ctas_res, ctas_tan64, ctas_tan32, order;
    double residual_ms, tangent_fp64_ms, tangent_fp32_ms;
    int colour_order;
} igab_batch_tune_result;
int igab_batch_autotune(igab_batch *b, const double *U_dev, int what, int reps, igab_batch_tune_result *out);

/* ---- history Jacobians of the transient physics (no reference counterpart; the discrete
 * adjoint of the time stepping needs them): CSR values (the tangent's pattern) of
 * d R / d U_hist[level] at U and the context's history levels, level 1 (t_n) or 2 (t_{n-1});
 * Dirichlet rows are zero (R = U - g there does not depend on the history).  The
 * matrices are symmetric; apply their transpose with igab_adjoint_backward. */
int igab_history_jacobian_device(igab_ctx *ctx, const double *U_dev, void *vals_dev, int prec, int level);

/* ---- integrated densities (replaces src/iga_intdensity.c:10 `iga_intdensity`):
 * HH[i] = sum over elements and Gauss points of w * density_i(u) minus the Neumann
 * boundary integrals of the boundary density (phys/ge/density.c: 13 values -- energy,
 * stresses, volume fractions; phys/getime/density.c: 2 values -- energy at the
 * midpoint of history levels 1 and 2 plus kinetic energy, and the Neumann area).
 * u is U (level 0) for phys/ge and the context's history levels for phys/getime;
 * the traction is the context's Neumann values (igab_set_neumann_values).
 * igab_ndensity gives the count; igab_intdensity copies HH to the host,
 * igab_intdensity_device writes it to device memory on the context's stream.
 * Sums are taken in a fixed order: results are bitwise repeatable. */
int igab_ndensity(const igab_ctx *ctx, int *n);
int igab_intdensity(igab_ctx *ctx, const double *U_host, double *HH_host);
int igab_intdensity_device(igab_ctx *ctx, const double *U_dev, double *HH_dev);

/* ---- device-resident linear algebra on the tangent (no tangent leaves the GPU; stands in
 * for the PETSc KSP solve of the reference's Newton iteration, src/snes_init.c).
 * igab_spmv_device: y = K x on the context's CSR pattern (vals FP64 or FP32, x, y FP64).
 * igab_solve_device: x = K^-1 b by right-preconditioned BiCGStab, Jacobi preconditioner
 * diag(K) (1 where a diagonal entry is 0), x0 = 0, stopping when ||b - K x|| <=
 * max(rtol ||b||, atol) or after maxit iterations; all scalars stay on the device and
 * iterations run as CUDA-graph replays of 8 (the context needs a non-default stream).
 * Repeated solves give bitwise equal results. */
typedef struct {
    int iterations;        /* iterations run (0 when b = 0) */
    int converged;         /* 1 when the tolerance was met */
    double residual_norm;  /* ||b - K x|| of the recurrence at exit */
    double rhs_norm;       /* ||b|| */
} igab_solve_info;
int igab_spmv_device(igab_ctx *ctx, const void *vals_dev, int prec, const double *x_dev, double *y_dev);
int igab_solve_device(igab_ctx *ctx, const void *vals_dev, int prec, const double *b_dev, double *x_dev,
                      double rtol, double atol, int maxit, igab_solve_info *info);

/* ---- multigrid-preconditioned Krylov solve on the tangent (no reference counterpart;
 * stands in for the PETSc KSP of src/snes_init.c:24-39).  The fourth-order phys/ge tangent
 * defeats Jacobi-preconditioned Krylov methods on fine meshes; the preconditioner here is a
 * geometric multigrid V-cycle on nested spline spaces: every other interior knot removed per
 * level (elements per direction halved while even and >= 4, down to about 1,200 dofs),
 * prolongation by knot insertion, all levels' operators the tangent at the zero state with
 * the context's material and (averaged) element scales (symmetric positive definite for a
 * stable material, so the V-cycle is an SPD preconditioner whatever the current state),
 * Chebyshev smoothing (degree 3 in D^-1 K), the coarsest level by its inverse (Gauss-Jordan on the device).  The hierarchy
 * is built on the first call and rebuilt after igab_set_par_mat / igab_set_par_periodic /
 * igab_set_element_log_scale.  method: IGAB_KSP_MG_GMRES (right-preconditioned GMRES(50),
 * any nonsingular tangent) or IGAB_KSP_MG_CG (CG, symmetric positive definite tangents; a
 * non-positive curvature p.Kp returns IGAB_ERR_UNSUPPORTED).  x0 = 0, stop at
 * ||b - K x|| <= max(rtol ||b||, atol).
 * igab_solve_mg_levels: levels of the current hierarchy (0 before the first solve).
 * igab_mg_prolongation_1d: the 1-D knot-insertion matrix P ((n+2+m) x (n+2), row-major) that
 * maps the spline coefficients on coarse_knots (n elements, open, p = 2) to those on the knot
 * vector with the m ascending interior knots `inserted` added. */
int igab_solve_mg_device(igab_ctx *ctx, int method, const void *vals_dev, int prec, const double *b_dev,
                         double *x_dev, double rtol, double atol, int maxit, igab_solve_info *info);
int igab_solve_mg_levels(igab_ctx *ctx, int *levels);
int igab_mg_prolongation_1d(const double *coarse_knots, int n_coarse_elements, const double *inserted,
                            int n_inserted, double *P);

/* ---- Newton solve on the device (replaces the reference application's solver loop,
 * src/snes_solve.c:10-36, run with the SNES configuration of src/snes_init.c:8-47):
 * one-step Newton solves (NEWTONLS, backtracking line search of cubic order; abstol on
 * ||F||_2, rtol, stol) repeated until a step ends with a reason other than "maximum
 * iterations", or until ||F|| stagnates (|F_old - F_new| / F_old < stagnation, F_old =
 * 999 at the start; reported as DIVERGED_LINE_SEARCH, as the reference does).  The linear
 * solve of each step (stand-in for PETSc's GMRES + ASM) runs to ksp_rtol on the tangent
 * assembled in opts.prec: opts.ksp selects multigrid GMRES or CG (igab_solve_mg_device) or
 * the Jacobi BiCGStab of igab_solve_device; no residual or tangent leaves the GPU.  With
 * opts.use_graph each assembly is replayed from a CUDA graph held by the context (captured
 * on first use, re-captured when a pointer, the precision or a parameter or schedule
 * setting changes).  U_dev holds the initial guess and receives the solution; the context's
 * Neumann values and history levels are used as set.  fnorm_history / krylov_history
 * (either may be NULL) receive ||F|| and the Krylov iteration count of the first
 * history_cap subiterations.  verbose = 1 prints the reference's line per subiteration. */
enum igab_ksp_kind { IGAB_KSP_BICGSTAB = 0, IGAB_KSP_MG_CG = 1, IGAB_KSP_MG_GMRES = 2 };
enum igab_snes_reason {
    IGAB_SNES_CONVERGED_FNORM_ABS = 2, IGAB_SNES_CONVERGED_FNORM_RELATIVE = 3,
    IGAB_SNES_CONVERGED_SNORM_RELATIVE = 4, IGAB_SNES_DIVERGED_FNORM_NAN = -4,
    IGAB_SNES_DIVERGED_MAX_IT = -5, IGAB_SNES_DIVERGED_LINE_SEARCH = -6
};   /* PETSc's SNESConvergedReason numbering */
typedef struct {
    int prec;              /* tangent precision: IGAB_PREC_FP64, or IGAB_PREC_FP32 (inexact Newton) */
    double abstol;         /* 1e-10   SNESSetTolerances, src/snes_init.c:18 */
    double rtol;           /* 1e-20 */
    double stol;           /* 1e-20 */
    double stagnation;     /* 1e-6    src/snes_solve.c:29 */
    int max_subiter;       /* 10000   src/snes_solve.c:24 */
    double ksp_rtol;       /* 1e-5    PETSc's default KSP relative tolerance */
    int ksp_maxit;         /* 100000  iterations per linear solve */
    int ksp;               /* IGAB_KSP_MG_GMRES (default), IGAB_KSP_MG_CG (phys/ge; BiCGStab for a step whose
                              CG meets non-positive curvature) or IGAB_KSP_BICGSTAB (Jacobi BiCGStab,
                              always for phys/getime) */
    int verbose;           /* 0 */
    int fp64_polish;       /* 0; with prec FP32: once a step reduces ||F|| by less than 10x (the FP32
                              tangent's error limits the step), the remaining steps use the FP64 tangent */
    int use_graph;         /* 1: residual and tangent assemblies replayed from CUDA graphs */
} igab_newton_opts;
typedef struct {
    int iterations;          /* Newton steps taken */
    int reason;              /* igab_snes_reason of the last subiteration */
    int converged;           /* reason > 0 */
    int n_residual, n_tangent;
    int n_tangent_fp64;      /* tangents assembled in FP64 (all of them for prec FP64; the polish steps) */
    long krylov_iterations;  /* over all linear solves */
    double fnorm;            /* ||F||_2 at exit */
    double ms_residual, ms_tangent, ms_krylov, ms_total;   /* wall time by phase */
    long launches;           /* kernels launched */
} igab_newton_info;
void igab_newton_defaults(igab_newton_opts *opts);
int igab_newton_solve(igab_ctx *ctx, double *U_dev, const igab_newton_opts *opts, igab_newton_info *info,
                      double *fnorm_history, int *krylov_history, int history_cap);

/* ---- time stepping of the transient physics on the device (replaces the application's
 * step of example/ex1/main.c:48-56 -- initial guess U = U_hist[1], snes_solve, history
 * shift U_hist[2] <- U_hist[1] <- U -- repeated nsteps times).  Step n (0-based) solves at
 * t = (n + 1) dt, with the traction amplitude * sin(2 pi t) on the Neumann points of the
 * (face, order, dof) combination given and zero on the other combinations of the BC table,
 * by igab_newton_solve with opts.newton.  U_dev: U at t_0 on entry (history level 1), U at
 * t_nsteps on return; U_prev_dev: U at t_-1 (history level 2; NULL = zero).  dt = 0 takes
 * the physics' own time step (par_mat[7]).  The history shifts after every step; a step
 * whose Newton solve ends without convergence is counted in info (steps_converged).  On
 * return the context's history levels hold U at t_nsteps - 1 and t_nsteps - 2.  Optional
 * outputs: U_steps_host (nsteps x ndof: the state after every step) and step_info
 * (nsteps entries). */
typedef struct {
    int nsteps;
    double dt;
    double amplitude;      /* 0.01 */
    int face, order, dof;  /* 1, 0, 0: x-traction on x = 1 */
    igab_newton_opts newton;
} igab_transient_opts;
typedef struct {
    int steps;               /* steps run */
    int steps_converged;
    long newton_iterations, krylov_iterations;
    long n_residual, n_tangent;
    double ms_total;         /* wall time of the whole run */
    long launches;
} igab_transient_info;
void igab_transient_defaults(igab_transient_opts *opts);
int igab_transient_run(igab_ctx *ctx, const igab_transient_opts *opts, double *U_dev, const double *U_prev_dev,
                       double *U_steps_host, igab_newton_info *step_info, igab_transient_info *info);

/* ---- discrete adjoint of the time stepping (no reference counterpart), for the element
 * log-scales g of igab_set_element_log_scale (set by the caller; the scales in force are
 * used).  Steps n = 0 .. N-1 solve R_n(U_{n+1}; U_n, U_{n-1}, g) = 0 as igab_transient_run
 * does.  For an objective J(U_N):
 *   K_n^T lam_n = b_n,  b_n = dJ/dU_{n+1} - J1_{n+1}^T lam_{n+1} - J0_{n+2}^T lam_{n+2},
 *   dJ/dg = - sum_n lam_n . dR_n/dg,
 * K_n the FP64 tangent at U_{n+1}, J1 / J0 the history Jacobians (levels 1 and 2), b and
 * lam zero on the Dirichlet rows, each K^T lam = b (K symmetric) solved by the Jacobi
 * BiCGStab to opts.newton.ksp_rtol.  The forward pass keeps the states at checkpoints
 * every `every` steps (two states each); the backward pass recomputes each segment from
 * its checkpoint (the same solves, so the same states bit for bit) before sweeping it:
 * device memory O(N / every + every) states plus two FP64 value arrays.
 * igab_tadj_create: the pass's buffers.  igab_tadj_forward: the N steps from U_init_dev
 * (U at t_0) and U_prev_dev (U at t_-1; NULL = zero), U_N into U_final_dev.
 * igab_tadj_backward: dJ/dg into grad_dev (nel doubles, device) from dJ/dU_N (device),
 * after a forward pass.  igab_tadj_info: counts of the last passes. */
typedef struct igab_tadj igab_tadj;
typedef struct {
    int forward_steps, recomputed_steps, checkpoints;
    int forward_converged;            /* forward steps whose Newton solve converged */
    long krylov_iterations_backward;  /* over the adjoint solves */
    int adjoint_solves_converged, adjoint_solves;
    double ms_forward, ms_backward;
} igab_tadj_info_t;
int igab_tadj_create(igab_ctx *ctx, const igab_transient_opts *opts, int every, igab_tadj **out);
int igab_tadj_forward(igab_tadj *t, const double *U_init_dev, const double *U_prev_dev, double *U_final_dev);
int igab_tadj_backward(igab_tadj *t, const double *dJdU_dev, double *grad_dev);
int igab_tadj_info(const igab_tadj *t, igab_tadj_info_t *info);
void igab_tadj_destroy(igab_tadj *t);

/* ---- mesh refinement and solution files (mesh/nurbs/nurbs_knotinsert.c:7, src/ioutil.c:89, :126).
 * igab_knot_insert: refine the p = 2 control points of a field, in place in host memory
 * (U_universal[ndof * cp + dof], cp = (x nb1 + y) nb2 + z with nb = nelem + 2, or nelem
 * along a periodic direction), from nelem / 2^nref to nelem elements per direction by
 * inserting the mid-point of every knot span nref times; the array must hold the refined
 * size.  porder must be 2; nelem a positive multiple of 2^nref.  Runs on the given GPU;
 * its two device buffers stay allocated between calls (grown to the largest refined
 * field seen on that device) and calls in one process are serialised.
 * igab_knot_release: frees those buffers on the given device (no counterpart in the
 * reference); the next igab_knot_insert allocates them again.
 * igab_write_solution / igab_read_solution: history levels ihist0 .. ihist1 - 1 of U_hist
 * (ndof doubles each) to / from a raw file, level after level, in the universal dof order
 * of one rank (the reference's format). */
int igab_knot_insert(double *U_universal, const int nelem[3], int nref, int porder, int ndof,
                     const int bc_periodic[3], int device);
int igab_knot_release(int device);
int igab_write_solution(const char *fname, const double *U_hist, long ndof, int ihist0, int ihist1);
int igab_read_solution(const char *fname, double *U_hist, long ndof, int ihist0, int ihist1);

/* ---- residual for callers that cannot have the library allocate device memory.
 * No counterpart in the reference.  Same result as igab_residual, but U and R
 * are staged in a file-scope device array (2 x 8 MiB, held by every GPU that
 * loads the library) instead of context buffers obtained with cudaMalloc; a
 * call allocates nothing.  Meshes above 1,048,576 dofs are rejected
 * (IGAB_ERR_ARG).  All calls share the array: calls that overlap on the GPU
 * race.  Each call looks up the array's address in the current CUDA context
 * (cudaGetSymbolAddress, which allocates nothing). */
int igab_residual_noalloc(igab_ctx *ctx, const double *U_host, double *R_host);
/* device bytes the context holds for the host-pointer entry points (the U, R and
 * tangent-value staging that igab_residual, igab_tangent and igab_device_buffers
 * allocate on first use; 0 before then).  No counterpart in the reference; lets a
 * caller check that igab_residual_noalloc left the context without staging. */
int igab_staging_bytes(const igab_ctx *ctx, size_t *bytes);

#ifdef __cplusplus
}
#endif

#endif
