/* Single-rank MPI shim (TEST INFRASTRUCTURE): only the calls the reference's
 * CPU path makes (mpi/*.cpp).  One rank, so Sendrecv is a copy (the periodic
 * wrap) and Allreduce(MPI_IN_PLACE) is the identity. */
#ifndef SHIM_MPI_H
#define SHIM_MPI_H
#include <stddef.h>
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef struct { int dummy; } MPI_Status;
#define MPI_COMM_WORLD 0
#define MPI_DOUBLE 1
#define MPI_INT 2
#define MPI_SUM 1
#define MPI_IN_PLACE ((void*)1)
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#ifdef __cplusplus
extern "C" {
#endif
int MPI_Init(int* argc, char*** argv);
int MPI_Finalize(void);
int MPI_Comm_rank(MPI_Comm c, int* r);
int MPI_Comm_size(MPI_Comm c, int* s);
int MPI_Comm_split(MPI_Comm c, int color, int key, MPI_Comm* out);
int MPI_Comm_free(MPI_Comm* c);
int MPI_Barrier(MPI_Comm c);
double MPI_Wtime(void);
int MPI_Allreduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype t, MPI_Op op, MPI_Comm c);
int MPI_Sendrecv(const void* sendbuf, int sendcount, MPI_Datatype st, int dest, int sendtag, void* recvbuf,
                 int recvcount, MPI_Datatype rt, int source, int recvtag, MPI_Comm c, MPI_Status* status);
#ifdef __cplusplus
}
#endif
#endif
