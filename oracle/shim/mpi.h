/*
 * Single-rank stand-in for the MPI API, used only to link GALIC's reference C
 * sources into the CPU oracle.  It is test infrastructure: nothing in the
 * product library includes it.
 *
 * With one rank every collective GALIC issues (e.g. the response-grid
 * MPI_Allreduce of main.c:259-285) is a copy of the send buffer into the
 * receive buffer; point-to-point calls are never reached, because every
 * exchange loop in the reference skips the rank's own task
 * (e.g. forcetree.c:308-316, gravtree.c:280-303).  Datatype handles encode
 * the element size in bytes.
 */
#ifndef GALIC_ORACLE_MPI_SHIM_H
#define GALIC_ORACLE_MPI_SHIM_H
#include <stddef.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR, count; } MPI_Status;

#define MPI_COMM_WORLD 1
#define MPI_BYTE (1 | (1 << 8))
#define MPI_CHAR (1 | (2 << 8))
#define MPI_INT (4 | (3 << 8))
#define MPI_UNSIGNED (4 | (4 << 8))
#define MPI_FLOAT (4 | (5 << 8))
#define MPI_DOUBLE (8 | (6 << 8))
#define MPI_LONG (8 | (7 << 8))
#define MPI_LONG_LONG (8 | (8 << 8))
#define MPI_UNSIGNED_LONG_LONG (8 | (9 << 8))
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_IN_PLACE ((void *) 1)
#define MPI_STATUS_IGNORE ((MPI_Status *) 0)
#define MPI_STATUSES_IGNORE ((MPI_Status *) 0)
#define MPI_SUCCESS 0

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Abort(MPI_Comm comm, int code);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm *newcomm);
int MPI_Comm_free(MPI_Comm *comm);
int MPI_Type_size(MPI_Datatype t, int *size);
int MPI_Barrier(MPI_Comm comm);
double MPI_Wtime(void);
int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, MPI_Comm c);
int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, int root, MPI_Comm c);
int MPI_Bcast(void *b, int n, MPI_Datatype t, int root, MPI_Comm c);
int MPI_Allgather(const void *s, int sn, MPI_Datatype st, void *r, int rn, MPI_Datatype rt, MPI_Comm c);
int MPI_Allgatherv(const void *s, int sn, MPI_Datatype st, void *r, const int *rn, const int *displs,
                   MPI_Datatype rt, MPI_Comm c);
int MPI_Gather(const void *s, int sn, MPI_Datatype st, void *r, int rn, MPI_Datatype rt, int root, MPI_Comm c);
int MPI_Alltoall(const void *s, int sn, MPI_Datatype st, void *r, int rn, MPI_Datatype rt, MPI_Comm c);
int MPI_Alltoallv(const void *s, const int *sn, const int *sd, MPI_Datatype st, void *r, const int *rn,
                  const int *rd, MPI_Datatype rt, MPI_Comm c);
int MPI_Sendrecv(const void *s, int sn, MPI_Datatype st, int dest, int stag, void *r, int rn, MPI_Datatype rt,
                 int src, int rtag, MPI_Comm c, MPI_Status *status);
int MPI_Send(const void *b, int n, MPI_Datatype t, int dest, int tag, MPI_Comm c);
int MPI_Ssend(const void *b, int n, MPI_Datatype t, int dest, int tag, MPI_Comm c);
int MPI_Recv(void *b, int n, MPI_Datatype t, int src, int tag, MPI_Comm c, MPI_Status *status);
int MPI_Isend(const void *b, int n, MPI_Datatype t, int dest, int tag, MPI_Comm c, MPI_Request *req);
int MPI_Irecv(void *b, int n, MPI_Datatype t, int src, int tag, MPI_Comm c, MPI_Request *req);
int MPI_Waitall(int n, MPI_Request *req, MPI_Status *status);
#endif
