/* Minimal stand-in for <mpi.h> so that the reference's physics sources
 * (which include it only through confmpi.h) compile in a single process.
 * No MPI function is declared: the harness never links the MPI layer
 * (manager_*, worker_*, confmpi.c). */
#ifndef MBT_ORACLE_STUB_MPI_H
#define MBT_ORACLE_STUB_MPI_H
#define MPI_MAX_PROCESSOR_NAME 128
#endif
