/* Minimal stand-in for <mpi.h>: only the names the reference's solver header
 * needs to compile (include/parallel/mpi_comm.hpp).  No MPI call is made by the
 * single-GPU path the harness drives. */
#ifndef ZJ_REF_MPI_STUB_H
#define ZJ_REF_MPI_STUB_H
typedef int MPI_Comm;
typedef int MPI_Request;
typedef int MPI_Datatype;
typedef int MPI_Op;
#define MPI_COMM_WORLD 0
static inline int MPI_Barrier(MPI_Comm c) { (void)c; return 0; }
#endif
