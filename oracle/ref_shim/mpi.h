/* mpi.h -- TEST INFRASTRUCTURE ONLY.  A one-rank stand-in for the MPI calls the
 * reference's sources make (MPI_Init/Finalize, rank and size, Barrier, Allreduce,
 * Bcast, Reduce), so that they compile unchanged into oracle/_ref.  With one rank
 * every reduction is a copy of the send buffer and a broadcast does nothing.
 * Project-written; only the names and argument lists follow the MPI standard. */
#ifndef REF_SHIM_MPI_H
#define REF_SHIM_MPI_H

#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;

#define MPI_COMM_WORLD 0
#define MPI_DOUBLE 1
#define MPI_C_BOOL 2
#define MPI_INT 3
#define MPI_SUM 1
#define MPI_LOR 2
#define MPI_MAX 3

static inline size_t ref_mpi_size_of(MPI_Datatype t) {
  return t == MPI_DOUBLE ? sizeof(double) : t == MPI_C_BOOL ? sizeof(bool) : sizeof(int);
}
static inline int MPI_Init(int*, char***) { return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int* rank) { *rank = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm, int* size) { *size = 1; return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Allreduce(const void* send, void* recv, int count, MPI_Datatype t, MPI_Op, MPI_Comm) {
  if (send != recv) memmove(recv, send, (size_t)count * ref_mpi_size_of(t));
  return 0;
}
static inline int MPI_Reduce(const void* send, void* recv, int count, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
  if (send != recv) memmove(recv, send, (size_t)count * ref_mpi_size_of(t));
  return 0;
}
static inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return 0; }

#endif
