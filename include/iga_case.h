/*
 * iga_case.h -- single-rank case builder for the SNES assembly callbacks.
 *
 * Builds the Phys / Nurbs / BC / IGA / SNESAssmbl / IOcomm objects for one
 * rank from plain arrays (the work nurbs_genuniform + nurbs_init + bc_init do
 * in IGAP4STANDARD: mesh/nurbs/nurbs_genuniform.c:8-52,
 * mesh/nurbs/nurbs_init.c:61-121, example/ex1/main.c:69-95), then calls
 * snesiga_init (src/snesiga_init.c:12) and drives the installed residual and
 * tangent callbacks exactly as SNESSolve would.  Arbitrary element counts
 * and arbitrary (e.g. perturbed) open knot vectors are accepted, which
 * nurbs_genuniform cannot express.
 *
 * The same source is linked against libsnesiga_b200 (GPU callbacks) and,
 * for the CPU oracle, against the reference's own callbacks; whichever
 * snesiga_init is linked decides which callbacks run.
 */
#ifndef IGA_CASE_H
#define IGA_CASE_H

#ifdef __cplusplus
extern "C" {
#endif

enum { IGA_CASE_GE = 0, IGA_CASE_GETIME = 1 };

typedef struct iga_case iga_case;

/* knots: the three open knot vectors back to back, nelem[d]+5 values each (p=2).
 * bc_type: 36 ints [face][order][dof]; par_*: 9 doubles each;
 * par_neumann: n_par_neumann doubles handed to neumann().  Returns NULL on error. */
iga_case *iga_case_create(int phys_kind, const int nelem[3], const double *knots,
                          const double par_mat[9], const int bc_type[36],
                          const double par_periodic[9], const double par_dirichlet[9],
                          const double *par_neumann, int n_par_neumann);
/* the same with periodic directions (bc_periodic[d] = 1): the knot vector of such a
 * direction is the uniform extension of mesh/nurbs/nurbs_genuniform.c:40-43 (nelem[d]+5
 * values), the rank owns nelem[d] points along it and exchanges the two ghost layers
 * with itself (mesh/nurbs/nurbs_init.c:24-39, :156-199 with npart = 1). */
iga_case *iga_case_create_periodic(int phys_kind, const int nelem[3], const double *knots,
                                   const double par_mat[9], const int bc_type[36],
                                   const double par_periodic[9], const double par_dirichlet[9],
                                   const double *par_neumann, int n_par_neumann, const int bc_periodic[3]);
/* the rank's index maps as snesiga_init left them (src/snesiga_init.c:42-50, :84-110):
 * counts into n[3] = {nselfIdx, nsendIdx, nrecvIdx}; arrays (either may be NULL) of
 * nselfIdx, nsendIdx, nrecvIdx and nselfIdx + nrecvIdx ints */
int  iga_case_index_maps(const iga_case *c, int n[3], int *selfIdx, int *sendIdx, int *recvIdx, int *globalIdx);
void iga_case_destroy(iga_case *c);

int  iga_case_ndof(const iga_case *c);
/* set history level `level` (1..torder) of U_hist, length ndof */
int  iga_case_set_history(iga_case *c, int level, const double *U);
int  iga_case_get_history(const iga_case *c, int level, double *U);
/* update parameters between calls (e.g. a time-dependent traction) */
int  iga_case_set_par_neumann(iga_case *c, const double *par_neumann, int n);
int  iga_case_set_par_dirichlet(iga_case *c, const double par_dirichlet[9]);
int  iga_case_set_par_mat(iga_case *c, const double par_mat[9]);

/* R = residual(U) through app->snes_Residual; returns its PetscErrorCode,
 * or the Vec/Mat error latch when the callback ignored an error. */
int  iga_case_residual(iga_case *c, const double *U, double *R);
/* tangent(U) into the case's AIJ matrix through app->snes_Tangent */
int  iga_case_tangent(iga_case *c, const double *U);
/* CSR of the assembled tangent: nnz first, then the arrays (caller-sized) */
long iga_case_tangent_nnz(const iga_case *c);
int  iga_case_tangent_csr(const iga_case *c, int *rowptr, int *cols, double *vals);

/* the library's solver loop (snes_solve, src/snes_solve.c:10) from the initial guess U;
 * U receives the solution.  0 converged, 1 not converged, -1 no snes_solve linked
 * (the oracle build has none: the reference's needs PETSc's SNES). */
int  iga_case_solve(iga_case *c, double *U);

/* opaque handles for code that wants to call further library functions */
void *iga_case_app(iga_case *c);
/* the IOcomm the case's snesiga_init filled (write_solution / read_solution, src/ioutil.c:89) */
void *iga_case_iocomm(iga_case *c);
void *iga_case_snesassmbl(iga_case *c);

/* the default app hook: neumann_ = par_neumann[6*face+3*order+idof]
 * * (1 + par_neumann[36]*x + par_neumann[37]*y + par_neumann[38]*z),
 * the last three read only when n_par_neumann >= 39. */
void iga_case_neumann(double *neumann_, double par_neumann[], int face_id, int bc_order, int idof, double xq[]);

#ifdef __cplusplus
}
#endif

#endif
