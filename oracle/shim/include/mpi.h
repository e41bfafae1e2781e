/* Single-rank stand-in for the MPI calls the frehg2 groundwater sources make.
 * Test infrastructure for compiling the reference's own sources on a host
 * without MPI: every communicator has exactly one rank, point-to-point calls
 * only ever target MPI_PROC_NULL (which MPI defines as a no-op), and
 * reductions copy their input to their output.  Any attempt to talk to a
 * real peer aborts loudly. */
#ifndef FREHG_SHIM_MPI_H
#define FREHG_SHIM_MPI_H

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 1
#define MPI_COMM_SELF 2
#define MPI_COMM_NULL 0
#define MPI_PROC_NULL (-2)
#define MPI_UNDEFINED (-32766)
#define MPI_REQUEST_NULL 0
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)
#define MPI_SUCCESS 0
#define MPI_THREAD_FUNNELED 1
#define MPI_MAX_PROCESSOR_NAME 256

#define MPI_CHAR 1
#define MPI_INT 4
#define MPI_LONG 8
#define MPI_LONG_LONG 9
#define MPI_DOUBLE 10
#define MPI_UNSIGNED_LONG 11
#define MPI_C_BOOL 12
#define MPI_BYTE 13
#define MPI_UNSIGNED 14
#define MPI_FLOAT 15
#define MPI_INT64_T 16

#define MPI_SUM 1
#define MPI_MIN 2
#define MPI_MAX 3
#define MPI_LOR 4
#define MPI_LAND 5

static inline size_t frehg_shim_mpi_size(MPI_Datatype t) {
  switch (t) {
    case MPI_CHAR: case MPI_BYTE: case MPI_C_BOOL: return 1;
    case MPI_INT: case MPI_UNSIGNED: case MPI_FLOAT: return 4;
    default: return 8;
  }
}
static inline void frehg_shim_mpi_peer(int peer) {
  if (peer != MPI_PROC_NULL) {
    fprintf(stderr, "single-rank MPI shim: point-to-point with rank %d\n", peer);
    abort();
  }
}

static inline int MPI_Init(int*, char***) { return 0; }
static inline int MPI_Init_thread(int*, char***, int, int* provided) {
  if (provided) *provided = MPI_THREAD_FUNNELED;
  return 0;
}
static inline int MPI_Initialized(int* flag) { *flag = 1; return 0; }
static inline int MPI_Finalized(int* flag) { *flag = 0; return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Abort(MPI_Comm, int code) { exit(code); }
static inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return 0; }
static inline int MPI_Comm_split(MPI_Comm c, int color, int, MPI_Comm* out) {
  *out = (color == MPI_UNDEFINED) ? MPI_COMM_NULL : c;
  return 0;
}
static inline int MPI_Comm_dup(MPI_Comm c, MPI_Comm* out) { *out = c; return 0; }
static inline int MPI_Comm_free(MPI_Comm* c) { *c = MPI_COMM_NULL; return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Dims_create(int nnodes, int ndims, int* dims) {
  for (int d = 0; d < ndims; ++d) {
    if (dims[d] == 0) dims[d] = 1;
  }
  (void)nnodes;
  return 0;
}
static inline int MPI_Allreduce(const void* in, void* out, int n, MPI_Datatype t, MPI_Op,
                                MPI_Comm) {
  if (in != out) memmove(out, in, (size_t)n * frehg_shim_mpi_size(t));
  return 0;
}
static inline int MPI_Reduce(const void* in, void* out, int n, MPI_Datatype t, MPI_Op, int,
                             MPI_Comm) {
  if (in != out && out) memmove(out, in, (size_t)n * frehg_shim_mpi_size(t));
  return 0;
}
static inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return 0; }
/* MPI_Exscan leaves rank 0's output undefined; callers overwrite it. */
static inline int MPI_Exscan(const void*, void*, int, MPI_Datatype, MPI_Op, MPI_Comm) {
  return 0;
}
static inline int MPI_Gather(const void* in, int n, MPI_Datatype t, void* out, int, MPI_Datatype,
                             int, MPI_Comm) {
  if (out) memmove(out, in, (size_t)n * frehg_shim_mpi_size(t));
  return 0;
}
static inline int MPI_Gatherv(const void* in, int n, MPI_Datatype t, void* out, const int*,
                              const int* displs, MPI_Datatype, int, MPI_Comm) {
  if (out) memmove((char*)out + (displs ? (size_t)displs[0] * frehg_shim_mpi_size(t) : 0), in,
                   (size_t)n * frehg_shim_mpi_size(t));
  return 0;
}
static inline int MPI_Allgather(const void* in, int n, MPI_Datatype t, void* out, int,
                                MPI_Datatype, MPI_Comm) {
  memmove(out, in, (size_t)n * frehg_shim_mpi_size(t));
  return 0;
}
static inline int MPI_Sendrecv(const void*, int, MPI_Datatype, int dst, int, void*, int,
                               MPI_Datatype, int src, int, MPI_Comm, MPI_Status*) {
  frehg_shim_mpi_peer(dst);
  frehg_shim_mpi_peer(src);
  return 0;
}
static inline int MPI_Isend(const void*, int, MPI_Datatype, int dst, int, MPI_Comm,
                            MPI_Request* r) {
  frehg_shim_mpi_peer(dst);
  *r = MPI_REQUEST_NULL;
  return 0;
}
static inline int MPI_Irecv(void*, int, MPI_Datatype, int src, int, MPI_Comm, MPI_Request* r) {
  frehg_shim_mpi_peer(src);
  *r = MPI_REQUEST_NULL;
  return 0;
}
static inline int MPI_Send(const void*, int, MPI_Datatype, int dst, int, MPI_Comm) {
  frehg_shim_mpi_peer(dst);
  return 0;
}
static inline int MPI_Recv(void*, int, MPI_Datatype, int src, int, MPI_Comm, MPI_Status*) {
  frehg_shim_mpi_peer(src);
  return 0;
}
static inline int MPI_Wait(MPI_Request*, MPI_Status*) { return 0; }
static inline int MPI_Waitall(int, MPI_Request*, MPI_Status*) { return 0; }
static inline double MPI_Wtime(void) { return 0.0; }
static inline int MPI_Get_processor_name(char* name, int* len) {
  strcpy(name, "localhost");
  *len = 9;
  return 0;
}

#endif /* FREHG_SHIM_MPI_H */
