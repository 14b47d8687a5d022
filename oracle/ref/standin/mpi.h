/* ORACLE — test infrastructure only.  A single-rank stand-in for the MPI
 * calls CUP2D's Poisson path makes (source/Poisson/{ExpAMRSolver.cpp,
 * LocalSpMatDnVec.cpp,BiCGSTAB.cu}, source/Utils/DeviceProfiler.cuh,
 * source/SimulationData.h): rank 0 of a world of 1.  Collectives copy the
 * send buffer to the receive buffer (MPI_IN_PLACE leaves it), which is what
 * MPI does on one rank; point-to-point calls are only ever posted to other
 * ranks by that code, so with one rank they are never reached and complete
 * immediately here. */
#ifndef CUP2D_ORACLE_MPI_STANDIN_H
#define CUP2D_ORACLE_MPI_STANDIN_H

#include <stddef.h>
#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct MPI_Status { int source, tag, error; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_CHAR 1
#define MPI_INT 2
#define MPI_LONG 3
#define MPI_LONG_LONG 4
#define MPI_FLOAT 5
#define MPI_DOUBLE 6
#define MPI_LONG_DOUBLE 7
#define MPI_UNSIGNED_LONG_LONG 8
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)
#define MPI_IN_PLACE ((void*)1)
#define MPI_THREAD_MULTIPLE 3

static inline size_t cup2d_mpi_standin_size(MPI_Datatype t) {
  switch (t) {
    case MPI_CHAR: return 1;
    case MPI_INT: return sizeof(int);
    case MPI_LONG: return sizeof(long);
    case MPI_LONG_LONG: return sizeof(long long);
    case MPI_UNSIGNED_LONG_LONG: return sizeof(unsigned long long);
    case MPI_FLOAT: return sizeof(float);
    case MPI_DOUBLE: return sizeof(double);
    case MPI_LONG_DOUBLE: return sizeof(long double);
    default: return 0;
  }
}

static inline int MPI_Comm_rank(MPI_Comm c, int* r) { (void)c; *r = 0; return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm c, int* s) { (void)c; *s = 1; return MPI_SUCCESS; }

static inline int MPI_Allreduce(const void* send, void* recv, int n, MPI_Datatype t, MPI_Op op, MPI_Comm c) {
  (void)op; (void)c;
  if (send != MPI_IN_PLACE) memcpy(recv, send, (size_t)n * cup2d_mpi_standin_size(t));
  return MPI_SUCCESS;
}

static inline int MPI_Allgather(const void* send, int ns, MPI_Datatype ts, void* recv, int nr, MPI_Datatype tr,
                                MPI_Comm c) {
  (void)nr; (void)tr; (void)c;
  if (send != MPI_IN_PLACE) memcpy(recv, send, (size_t)ns * cup2d_mpi_standin_size(ts));
  return MPI_SUCCESS;
}

static inline int MPI_Alltoall(const void* send, int ns, MPI_Datatype ts, void* recv, int nr, MPI_Datatype tr,
                               MPI_Comm c) {
  (void)nr; (void)tr; (void)c;
  if (send != MPI_IN_PLACE) memcpy(recv, send, (size_t)ns * cup2d_mpi_standin_size(ts));
  return MPI_SUCCESS;
}

static inline int MPI_Isend(const void* b, int n, MPI_Datatype t, int dst, int tag, MPI_Comm c, MPI_Request* r) {
  (void)b; (void)n; (void)t; (void)dst; (void)tag; (void)c;
  *r = 0;
  return MPI_SUCCESS;
}

static inline int MPI_Irecv(void* b, int n, MPI_Datatype t, int src, int tag, MPI_Comm c, MPI_Request* r) {
  (void)b; (void)n; (void)t; (void)src; (void)tag; (void)c;
  *r = 0;
  return MPI_SUCCESS;
}

static inline int MPI_Waitall(int n, MPI_Request* r, MPI_Status* s) { (void)n; (void)r; (void)s; return MPI_SUCCESS; }
static inline int MPI_Barrier(MPI_Comm c) { (void)c; return MPI_SUCCESS; }

#endif
