// Test stand-in for the MPI calls the metad-b200 shim makes; the harness
// implements them over host threads, one thread per rank.
#ifndef STUB_MPI_H
#define STUB_MPI_H
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
#define MPI_SUCCESS 0
#define MPI_DOUBLE 1
#define MPI_SUM 1
#define MPI_IN_PLACE ((void *) 1)
int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype type, MPI_Op op, MPI_Comm comm);
#endif
