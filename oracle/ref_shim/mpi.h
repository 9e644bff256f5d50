/* Test-infrastructure shim: lets the reference's tree/walk sources
 * (src/fmm.c, src/global.c, src/operator.c, src/memory.c) compile on a host
 * without MPI. Only the type names those files mention are provided; no MPI
 * call is reachable from the oracle harness. */
#ifndef PHOTONS_ORACLE_MPI_SHIM_H
#define PHOTONS_ORACLE_MPI_SHIM_H
typedef int MPI_Datatype;
typedef int MPI_Comm;
typedef int MPI_Status;
typedef int MPI_Request;
#define MPI_COMM_WORLD 0
#endif
