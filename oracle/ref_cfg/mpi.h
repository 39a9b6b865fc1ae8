/* Test infrastructure only.  Stand-in for <mpi.h> in the serial build of
 * the reference (src/bfam.h includes <mpi.h>): the MPI names the reference
 * uses, mapped to libsc's single-process sc_MPI_* replacements. */
#ifndef BFAM_ORACLE_MPI_SHIM_H
#define BFAM_ORACLE_MPI_SHIM_H
#include <sc.h>
#include <string.h>
#define MPI_SUCCESS sc_MPI_SUCCESS
#define MPI_Comm sc_MPI_Comm
#define MPI_COMM_WORLD sc_MPI_COMM_WORLD
#define MPI_COMM_NULL sc_MPI_COMM_NULL
#define MPI_Request sc_MPI_Request
#define MPI_REQUEST_NULL sc_MPI_REQUEST_NULL
#define MPI_Status sc_MPI_Status
#define MPI_BYTE sc_MPI_BYTE
#define MPI_CHAR sc_MPI_CHAR
#define MPI_INT sc_MPI_INT
#define MPI_LONG_LONG_INT sc_MPI_LONG_LONG_INT
#define MPI_FLOAT sc_MPI_FLOAT
#define MPI_DOUBLE sc_MPI_DOUBLE
#define MPI_SUM sc_MPI_SUM
#define MPI_MAX_PROCESSOR_NAME 64
#define MPI_Comm_rank sc_MPI_Comm_rank
#define MPI_Comm_size sc_MPI_Comm_size
#define MPI_Allgather sc_MPI_Allgather
#define MPI_Reduce sc_MPI_Reduce
#define MPI_Irecv sc_MPI_Irecv
#define MPI_Isend sc_MPI_Isend
#define MPI_Waitall sc_MPI_Waitall
#define MPI_Wtime sc_MPI_Wtime
static inline int MPI_Get_processor_name(char *name, int *len)
{
  strcpy(name, "localhost");
  *len = (int)strlen(name);
  return sc_MPI_SUCCESS;
}
#endif
