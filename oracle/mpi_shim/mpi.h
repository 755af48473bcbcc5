/*
 * Single-rank stand-in for the MPI interface, used only to build the
 * reference ECOGEN sources as a serial CPU oracle (test infrastructure).
 *
 * ECOGEN calls MPI for rank/size, barriers, reductions of one value
 * (dt MIN, error SUM, pMax MAX), gathers for AMR balancing and persistent
 * point-to-point halo exchanges (src/Parallel/Parallel.cpp:243-405).  With a
 * single rank every reduction and gather is a copy and no point-to-point
 * message is ever posted, so this header implements exactly that.
 */
#ifndef ECG_ORACLE_MPI_SHIM_H
#define ECG_ORACLE_MPI_SHIM_H

#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
/* datatype codes carry the element size in bytes */
#define MPI_INT ((MPI_Datatype)sizeof(int))
#define MPI_DOUBLE ((MPI_Datatype)sizeof(double))
#define MPI_C_BOOL ((MPI_Datatype)sizeof(bool))
#define MPI_UNSIGNED_LONG_LONG ((MPI_Datatype)sizeof(unsigned long long))
#define MPI_MIN 1
#define MPI_MAX 2
#define MPI_SUM 3

static inline int MPI_Init(int*, char***) { return 0; }
static inline int MPI_Finalize() { return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Allreduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
  if (s != r) memmove(r, s, (size_t)n * (size_t)t);
  return 0;
}
static inline int MPI_Allgather(const void* s, int n, MPI_Datatype t, void* r, int, MPI_Datatype, MPI_Comm) {
  if (s != r) memmove(r, s, (size_t)n * (size_t)t);
  return 0;
}
static inline int MPI_Allgatherv(const void* s, int n, MPI_Datatype t, void* r, const int*, const int* displs,
                                 MPI_Datatype, MPI_Comm) {
  memmove((char*)r + (size_t)displs[0] * (size_t)t, s, (size_t)n * (size_t)t);
  return 0;
}
static inline int MPI_Send_init(const void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request* q) { *q = 0; return 0; }
static inline int MPI_Recv_init(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request* q) { *q = 0; return 0; }
static inline int MPI_Isend(const void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request* q) { *q = 0; return 0; }
static inline int MPI_Irecv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request* q) { *q = 0; return 0; }
static inline int MPI_Start(MPI_Request*) { return 0; }
static inline int MPI_Wait(MPI_Request*, MPI_Status*) { return 0; }
static inline int MPI_Request_free(MPI_Request*) { return 0; }

#endif
