/* Single-rank implementation of the MPI calls GALIC's reference sources make.
 * Test infrastructure for the CPU oracle only.  See mpi.h. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include "mpi.h"

static size_t esize(MPI_Datatype t) { return (size_t) (t & 0xff); }
static void copy(const void *s, void *r, size_t bytes)
{
  if(s != MPI_IN_PLACE && s != r && bytes) memmove(r, s, bytes);
}
static int unreachable(const char *what)
{
  fprintf(stderr, "oracle MPI stand-in: %s needs a second rank\n", what);
  abort();
  return 1;
}

int MPI_Init(int *argc, char ***argv) { (void) argc; (void) argv; return 0; }
int MPI_Finalize(void) { return 0; }
int MPI_Abort(MPI_Comm comm, int code) { (void) comm; fflush(stdout); exit(code ? code : 1); }
int MPI_Comm_rank(MPI_Comm comm, int *rank) { (void) comm; *rank = 0; return 0; }
int MPI_Comm_size(MPI_Comm comm, int *size) { (void) comm; *size = 1; return 0; }
int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm *nc) { (void) color; (void) key; *nc = comm; return 0; }
int MPI_Comm_free(MPI_Comm *comm) { (void) comm; return 0; }
int MPI_Type_size(MPI_Datatype t, int *size) { *size = (int) esize(t); return 0; }
int MPI_Barrier(MPI_Comm comm) { (void) comm; return 0; }
double MPI_Wtime(void)
{
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}
int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, MPI_Comm c)
{ (void) op; (void) c; copy(s, r, n * esize(t)); return 0; }
int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, int root, MPI_Comm c)
{ (void) op; (void) root; (void) c; copy(s, r, n * esize(t)); return 0; }
int MPI_Bcast(void *b, int n, MPI_Datatype t, int root, MPI_Comm c)
{ (void) b; (void) n; (void) t; (void) root; (void) c; return 0; }
int MPI_Allgather(const void *s, int sn, MPI_Datatype st, void *r, int rn, MPI_Datatype rt, MPI_Comm c)
{ (void) rn; (void) rt; (void) c; copy(s, r, sn * esize(st)); return 0; }
int MPI_Allgatherv(const void *s, int sn, MPI_Datatype st, void *r, const int *rn, const int *displs,
                   MPI_Datatype rt, MPI_Comm c)
{ (void) rn; (void) c; copy(s, (char *) r + displs[0] * esize(rt), sn * esize(st)); return 0; }
int MPI_Gather(const void *s, int sn, MPI_Datatype st, void *r, int rn, MPI_Datatype rt, int root, MPI_Comm c)
{ (void) rn; (void) rt; (void) root; (void) c; copy(s, r, sn * esize(st)); return 0; }
int MPI_Alltoall(const void *s, int sn, MPI_Datatype st, void *r, int rn, MPI_Datatype rt, MPI_Comm c)
{ (void) rn; (void) rt; (void) c; copy(s, r, sn * esize(st)); return 0; }
int MPI_Alltoallv(const void *s, const int *sn, const int *sd, MPI_Datatype st, void *r, const int *rn,
                  const int *rd, MPI_Datatype rt, MPI_Comm c)
{
  (void) rn; (void) c;
  copy((const char *) s + sd[0] * esize(st), (char *) r + rd[0] * esize(rt), sn[0] * esize(st));
  return 0;
}
int MPI_Sendrecv(const void *s, int sn, MPI_Datatype st, int dest, int stag, void *r, int rn, MPI_Datatype rt,
                 int src, int rtag, MPI_Comm c, MPI_Status *status)
{
  (void) stag; (void) rn; (void) rt; (void) rtag; (void) c; (void) status;
  if(dest != 0 || src != 0) return unreachable("MPI_Sendrecv");
  copy(s, r, sn * esize(st));
  return 0;
}
int MPI_Send(const void *b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c)
{ (void) b; (void) n; (void) t; (void) d; (void) tag; (void) c; return unreachable("MPI_Send"); }
int MPI_Ssend(const void *b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c)
{ (void) b; (void) n; (void) t; (void) d; (void) tag; (void) c; return unreachable("MPI_Ssend"); }
int MPI_Recv(void *b, int n, MPI_Datatype t, int s, int tag, MPI_Comm c, MPI_Status *st)
{ (void) b; (void) n; (void) t; (void) s; (void) tag; (void) c; (void) st; return unreachable("MPI_Recv"); }
int MPI_Isend(const void *b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c, MPI_Request *rq)
{ (void) b; (void) n; (void) t; (void) d; (void) tag; (void) c; (void) rq; return unreachable("MPI_Isend"); }
int MPI_Irecv(void *b, int n, MPI_Datatype t, int s, int tag, MPI_Comm c, MPI_Request *rq)
{ (void) b; (void) n; (void) t; (void) s; (void) tag; (void) c; (void) rq; return unreachable("MPI_Irecv"); }
int MPI_Waitall(int n, MPI_Request *rq, MPI_Status *st) { (void) n; (void) rq; (void) st; return 0; }
