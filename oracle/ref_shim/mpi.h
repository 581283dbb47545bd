/* Compile-only stand-in for <mpi.h> used when building the reference's
 * single-process search path as a test oracle.  Every function aborts: the
 * ORIGINAL search mode and a directly driven BaseWorker never reach MPI. */
#pragma once
#include <cstdio>
#include <cstdlib>
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE; int MPI_TAG; int MPI_ERROR; } MPI_Status;
#define MPI_COMM_WORLD 0
#define MPI_BYTE 1
#define MPI_FLOAT 2
#define MPI_DOUBLE 3
#define MPI_INT64_T 4
#define MPI_TAG_UB 5
#define MPI_THREAD_MULTIPLE 3
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)
[[noreturn]] inline int oracle_mpi_unreachable(const char* f) {
  std::fprintf(stderr, "oracle: MPI call %s is not available in the single-process oracle\n", f);
  std::abort();
}
#define ORACLE_MPI_FN(name) template <typename... A> inline int name(A...) { oracle_mpi_unreachable(#name); }
ORACLE_MPI_FN(MPI_Abort)
ORACLE_MPI_FN(MPI_Barrier)
ORACLE_MPI_FN(MPI_Bcast)
ORACLE_MPI_FN(MPI_Comm_get_attr)
ORACLE_MPI_FN(MPI_Irecv)
ORACLE_MPI_FN(MPI_Isend)
ORACLE_MPI_FN(MPI_Recv)
ORACLE_MPI_FN(MPI_Send)
ORACLE_MPI_FN(MPI_Test)
ORACLE_MPI_FN(MPI_Wait)
ORACLE_MPI_FN(MPI_Waitall)
ORACLE_MPI_FN(MPI_Init_thread)
ORACLE_MPI_FN(MPI_Comm_rank)
ORACLE_MPI_FN(MPI_Comm_size)
ORACLE_MPI_FN(MPI_Finalize)
