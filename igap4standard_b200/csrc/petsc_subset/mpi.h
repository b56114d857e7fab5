/*
 * Single-rank MPI subset.
 *
 * The element-assembly callbacks of IGAP4STANDARD only talk to MPI for the
 * upper-ghost halo of U (src/snesiga_Residual.c:61-72, src/snesiga_Tangent.c:61-72),
 * for the setup-time index maps (src/snesiga_init.c:57-104) and for the knot
 * partition (mesh/nurbs/nurbs_init.c:190-194).  On one rank every collective
 * is a copy and every point-to-point message goes to this same rank.  This
 * header gives exactly that, so the assembly code (ours, and the reference's
 * compiled for the CPU oracle) builds and runs where no MPI is installed.  A
 * build against a real MPI simply puts the real mpi.h first on the include
 * path; nothing else changes.
 */
#ifndef IGAB_MPI_SUBSET_H
#define IGAB_MPI_SUBSET_H

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE; int MPI_TAG; int MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD ((MPI_Comm)0)
#define MPI_COMM_SELF  ((MPI_Comm)1)
#define MPI_SUCCESS    0
#define MPI_ERR_OTHER  15

#define MPI_INT    ((MPI_Datatype)1)
#define MPI_DOUBLE ((MPI_Datatype)2)
#define MPI_CHAR   ((MPI_Datatype)3)

#define MPI_SUM ((MPI_Op)1)
#define MPI_MAX ((MPI_Op)2)
#define MPI_MIN ((MPI_Op)3)

#define MPI_STATUS_IGNORE ((MPI_Status *)0)

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Isend(const void *buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm, MPI_Request *req);
int MPI_Irecv(void *buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm comm, MPI_Request *req);
int MPI_Wait(MPI_Request *req, MPI_Status *status);
int MPI_Gather(const void *sbuf, int scount, MPI_Datatype stype, void *rbuf, int rcount, MPI_Datatype rtype, int root, MPI_Comm comm);
int MPI_Gatherv(const void *sbuf, int scount, MPI_Datatype stype, void *rbuf, const int *rcounts, const int *displs, MPI_Datatype rtype, int root, MPI_Comm comm);
int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root, MPI_Comm comm);
int MPI_Scatter(const void *sbuf, int scount, MPI_Datatype stype, void *rbuf, int rcount, MPI_Datatype rtype, int root, MPI_Comm comm);
int MPI_Scatterv(const void *sbuf, const int *scounts, const int *displs, MPI_Datatype stype, void *rbuf, int rcount, MPI_Datatype rtype, int root, MPI_Comm comm);
int MPI_Allreduce(const void *sbuf, void *rbuf, int count, MPI_Datatype type, MPI_Op op, MPI_Comm comm);
int MPI_Barrier(MPI_Comm comm);

#ifdef __cplusplus
}
#endif

#endif
