/*
 * Single-rank stand-in for the MPI API used by the reference sources, so that its solver
 * files compile unmodified for one process (test infrastructure: the reference harness only).
 * Collectives copy the send buffer, point-to-point with MPI_PROC_NULL does nothing, the
 * Cartesian topology is 1x1x1.
 */
#ifndef CGFD_REF_SHIM_MPI_H
#define CGFD_REF_SHIM_MPI_H
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Request;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_PROC_NULL (-2)
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)
#define MPI_CHAR 1
#define MPI_INT 2
#define MPI_LONG 3
#define MPI_FLOAT 4
#define MPI_REAL 4
#define MPI_DOUBLE 5
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3

static inline size_t cgfd_shim_size(MPI_Datatype t) {
  switch (t) {
    case MPI_CHAR: return 1;
    case MPI_INT: return sizeof(int);
    case MPI_LONG: return sizeof(long);
    case MPI_FLOAT: return sizeof(float);
    case MPI_DOUBLE: return sizeof(double);
  }
  return 1;
}
static inline int MPI_Init(int *a, char ***b) { (void)a; (void)b; return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Abort(MPI_Comm c, int code) { (void)c; fprintf(stderr, "MPI_Abort(%d)\n", code); exit(code ? code : 1); }
static inline int MPI_Barrier(MPI_Comm c) { (void)c; return 0; }
static inline int MPI_Comm_rank(MPI_Comm c, int *r) { (void)c; *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm c, int *s) { (void)c; *s = 1; return 0; }
static inline int MPI_Bcast(void *b, int n, MPI_Datatype t, int root, MPI_Comm c) { (void)b; (void)n; (void)t; (void)root; (void)c; return 0; }
static inline int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, MPI_Comm c) {
  (void)op; (void)c;
  if (s != r) memmove(r, s, (size_t)n * cgfd_shim_size(t));
  return 0;
}
static inline int MPI_Allgather(const void *s, int ns, MPI_Datatype ts, void *r, int nr, MPI_Datatype tr, MPI_Comm c) {
  (void)nr; (void)tr; (void)c;
  memmove(r, s, (size_t)ns * cgfd_shim_size(ts));
  return 0;
}
static inline int MPI_Sendrecv(const void *sb, int sc, MPI_Datatype st, int dst, int stag, void *rb, int rc,
                               MPI_Datatype rt, int src, int rtag, MPI_Comm c, MPI_Status *s) {
  (void)sb; (void)sc; (void)st; (void)dst; (void)stag; (void)rb; (void)rc; (void)rt; (void)src; (void)rtag; (void)c; (void)s;
  return 0;
}
static inline int MPI_Type_vector(int n, int b, int s, MPI_Datatype o, MPI_Datatype *t) { (void)n; (void)b; (void)s; *t = o; return 0; }
static inline int MPI_Type_commit(MPI_Datatype *t) { (void)t; return 0; }
static inline int MPI_Send_init(const void *b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c, MPI_Request *r) {
  (void)b; (void)n; (void)t; (void)d; (void)tag; (void)c; *r = 0; return 0;
}
static inline int MPI_Recv_init(void *b, int n, MPI_Datatype t, int s, int tag, MPI_Comm c, MPI_Request *r) {
  (void)b; (void)n; (void)t; (void)s; (void)tag; (void)c; *r = 0; return 0;
}
static inline int MPI_Startall(int n, MPI_Request *r) { (void)n; (void)r; return 0; }
static inline int MPI_Waitall(int n, MPI_Request *r, MPI_Status *s) { (void)n; (void)r; (void)s; return 0; }
static inline int MPI_Cart_create(MPI_Comm o, int nd, const int *dims, const int *per, int re, MPI_Comm *c) {
  (void)o; (void)nd; (void)dims; (void)per; (void)re; *c = 0; return 0;
}
static inline int MPI_Cart_coords(MPI_Comm c, int rank, int nd, int *co) { (void)c; (void)rank; for (int i = 0; i < nd; i++) co[i] = 0; return 0; }
static inline int MPI_Cart_shift(MPI_Comm c, int d, int disp, int *s, int *t) { (void)c; (void)d; (void)disp; *s = MPI_PROC_NULL; *t = MPI_PROC_NULL; return 0; }
#endif
