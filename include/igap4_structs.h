/*
 * igap4_structs.h -- the host structs the SNES assembly callbacks receive.
 *
 * These declarations are binary-compatible with IGAP4STANDARD's own
 * (member order, types and meaning are the same; names too, because user
 * code fills them):
 *   Phys        include/phys.h:11-26   (physics plugin table)
 *   Nurbs       include/nurbs.h:4-24   (knot vectors, partition, boundary list)
 *   BC          include/bc.h:4-11      (bc_type table, affine/traction parameters)
 *   IGA         include/iga.h:8-25     (the `app` context handed to the callbacks)
 *   SNESAssmbl  include/snes.h:9-18    (callback pointers, Residual_/Tangent_/U)
 *   IOcomm      include/iocomm.h:4-11  (universal ordering for I/O)
 * A program that builds these structs for the reference library can hand
 * the same objects to libsnesiga_b200 without recompiling.
 */
#ifndef IGAP4_STRUCTS_H
#define IGAP4_STRUCTS_H

#include "petscsnes.h"

#ifdef __cplusplus
extern "C" {
#endif

/* integrand signatures: out[30] / out[900] from u[(torder+1)*30] and par[9] */
typedef void (*residual_ptr)(double *residual_, double *u, double *par);
typedef void (*tangent_ptr)(double *tangent_, double *u, double *par);
typedef void (*field_ptr)(double *field, double *u, double *par);
typedef void (*density_ptr)(double h[], double u[], double *par);
typedef void (*densityb_ptr)(double h[], double u[], double traction, double *par, int order);
typedef void (*assert_par_mat_ptr)(double *par);

typedef struct {
    int ndim;
    int ndof;
    int torder;
    int sorder;
    double *par_mat;
    int ndensity;
    int nfield;

    residual_ptr       residual;
    tangent_ptr        tangent;
    field_ptr          field;
    density_ptr        density;
    densityb_ptr       densityb;
    assert_par_mat_ptr assert_par_mat;
} Phys;

typedef struct {
    int porder;
    int *nelem;
    int *nbasis;
    int *nknot;
    double **knotVector;
    int nboun;
    int *boun;
    int nsendPart;
    int *sendPart;
    int nrecvPart;
    int *recvPart;
    int *sendBlock;
    int *recvBlock;
    int *universalIdx_temp;
    int *bc_periodic;
    int *nelem_global;
    double **knotVector_global;
} Nurbs;

typedef struct {
    int *bc_type;          /* [6 faces][2 orders][ndof]: 0 Dirichlet, 1 Neumann */
    double *par_periodic;  /* [ndof*ndim] affine F0 added to u at Gauss points */
    double *par_dirichlet; /* [ndof*ndim] affine map of the Dirichlet values */
    double *par_neumann;   /* app-defined, read only by neumann() */
} BC;

typedef struct {
    Phys  *phys;
    Nurbs *nurbs;
    BC    *bc;

    double *U_hist;
    int nselfIdx;
    int *selfIdx;
    int nsendIdx;
    int *sendIdx;
    int *sendPtr;
    int nrecvIdx;
    int *recvIdx;
    int *recvPtr;
    int *globalIdx;
} IGA;

typedef PetscErrorCode (*snes_Residual_ptr)(SNES, Vec, Vec, void *);
typedef PetscErrorCode (*snes_Tangent_ptr)(SNES, Vec, Mat, Mat, void *);

typedef struct {
    snes_Residual_ptr snes_Residual;
    snes_Tangent_ptr  snes_Tangent;
    Vec               Residual_;
    Mat               Tangent_;

    SNES              snes;
    Vec               U;
    int               converged;
} SNESAssmbl;

typedef struct {
    int nDof;
    int *nDof_array;
    int *iDof_displ_array;
    int nDof_global;
    int *universalIdx;
} IOcomm;

/* App-supplied hooks the assembly library calls (include/bc.h:13-14). */
void neumann(double *neumann_, double par_neumann[], int face_id, int bc_order, int idof, double xq[]);

#ifdef __cplusplus
}
#endif

#endif
