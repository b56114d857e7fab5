/*
 * snesiga_b200.h -- drop-in PETSc SNES callbacks backed by the B200 kernels
 * (libsnesiga_b200.so).
 *
 * Same names and signatures as IGAP4STANDARD's include/snesiga.h:8-11, so an
 * unmodified driver (snes_init registers app->snes_Residual/snes_Tangent,
 * src/snes_init.c:16-17) links against this library instead of libigap4's
 * assembly:
 *   snesiga_Residual  replaces src/snesiga_Residual.c:13   (same side effect:
 *                     U_hist[0..nselfIdx) <- U, :60)
 *   snesiga_Tangent   replaces src/snesiga_Tangent.c:13    (assembles into Pmat_,
 *                     assembles Tangent_ if it differs, :275-279)
 *   snesiga_init      replaces src/snesiga_init.c:12       (single rank)
 *   iga_intdensity    replaces src/iga_intdensity.c:10     (integrated densities)
 * The GPU state (device buffers, pattern check, traction table) lives in a
 * registry keyed by the IGA pointer, so the IGA struct stays binary-identical.
 * It is created on the first callback (or by snesiga_gpu_init) and released
 * by snesiga_gpu_free.
 *
 * Errors: where the reference asserts or exits, these return a nonzero
 * PetscErrorCode (PETSC_ERR_LIB for CUDA failures, PETSC_ERR_FP for a
 * non-finite residual or tangent, PETSC_ERR_SUP for unsupported physics or
 * more than one rank), so SNES sees the failure.
 */
#ifndef SNESIGA_B200_H
#define SNESIGA_B200_H

#include "igap4_structs.h"
#include "igab.h"

#ifdef __cplusplus
extern "C" {
#endif

PetscErrorCode snesiga_Residual(SNES snes, Vec U_, Vec Residual_, void *app_);
PetscErrorCode snesiga_Tangent(SNES snes, Vec U_, Mat Tangent_, Mat Pmat_, void *app_);
void snesiga_init(void *app_, void *phys_, void *nurbs_, void *bc_, void *snesassmbl_, void *iocomm_);

/* integrated densities of app->U_hist, replacing src/iga_intdensity.c:10
 * (include/iga.h:29); NaN in every slot on failure (the reference returns void) */
void iga_intdensity(double HH_[], void *app_);
/* knot-insertion refinement (mesh/nurbs/nurbs_knotinsert.c:7) and solution files
 * (src/ioutil.c:89, :126), same signatures; errors are printed (the reference asserts) */
void nurbs_knotinsert(double *U_universal, const int nelem[], int nref, int porder, int ndim, int ndof,
                      int bc_periodic[]);
void write_solution(const char *fname, double *U_hist, void *iocomm_, int ihist0, int ihist1);
void read_solution(const char *fname, double *U_hist, void *iocomm_, int ihist0, int ihist1);

/* the same callbacks under names that cannot collide with libigap4 */
PetscErrorCode snesiga_b200_Residual(SNES snes, Vec U_, Vec Residual_, void *app_);
PetscErrorCode snesiga_b200_Tangent(SNES snes, Vec U_, Mat Tangent_, Mat Pmat_, void *app_);
void snesiga_b200_intdensity(double HH_[], void *app_);

/* explicit GPU state management (optional; the callbacks create it lazily) */
PetscErrorCode snesiga_gpu_init(void *app_, int device);
PetscErrorCode snesiga_gpu_free(void *app_);
/* the traction hook to call at surface Gauss points (default: the `neumann`
 * symbol the application defines, include/bc.h:14) */
int snesiga_gpu_set_neumann(void *app_, void (*fn)(double *, double[], int, int, int, double[]));
/* when to re-evaluate the traction: 0 every residual call (default),
 * 1 only on the first call, 2 whenever the first `n_watch` doubles of
 * BC.par_neumann change */
int snesiga_gpu_set_neumann_policy(void *app_, int policy, int n_watch);
/* tangent arithmetic: 0 FP64 (default), 1 FP32 built and accumulated, widened on copy-out */
int snesiga_gpu_set_tangent_precision(void *app_, int prec);
/* the underlying igab context (include/igab.h), or NULL */
void *snesiga_gpu_context(void *app_);
/* milliseconds of the last callback: [0] residual total, [1] tangent total,
 * [2] residual kernels, [3] tangent kernels */
int snesiga_gpu_last_timings(void *app_, double ms[4]);

/* The solver loop on the GPU, replacing src/snes_solve.c:10 (same signature): the
 * Newton iteration of src/snes_init.c:8-47 / src/snes_solve.c:10-36 with every
 * residual, tangent and Krylov solve on the device (igab_newton_solve; the tangent
 * never reaches the host AIJ matrix).  Initial guess and solution in
 * snesassmbl->U; afterwards app->U_hist[0..nselfIdx) holds the solution and
 * snesassmbl->Residual_ the residual there; snesassmbl->converged is set.  Prints
 * the reference's line per subiteration.  The SNESAssmbl must come from this
 * library's snesiga_init.  Tangent precision: snesiga_gpu_set_tangent_precision. */
void snes_solve(void *snesassmbl_);
void snesiga_b200_solve(void *snesassmbl_);
/* Krylov tolerance and iteration limit of the device solve (0: defaults 1e-5, 100000) */
int snesiga_gpu_set_ksp(void *app_, double rtol, int maxit);
/* iteration counts, norms and phase times of the last snes_solve on this application */
int snesiga_gpu_last_solve(void *app_, igab_newton_info *info);

#ifdef __cplusplus
}
#endif

#endif
