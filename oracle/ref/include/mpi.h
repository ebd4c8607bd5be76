/* Single-rank stand-in for the MPI API, used only to link the reference
 * transport code into the oracle harness on a machine without MPI.
 * Test infrastructure: every collective is a local copy (one rank). */
#ifndef ORACLE_SHIM_MPI_H
#define ORACLE_SHIM_MPI_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;

#define MPI_COMM_WORLD 0
#define MPI_INT 1
#define MPI_DOUBLE 2
#define MPI_FLOAT 3
#define MPI_CHAR 4
#define MPI_UNSIGNED_LONG 5
#define MPI_LONG 6
#define MPI_SUM 0
#define MPI_MAX 1
#define MPI_MIN 2
#define MPI_IN_PLACE ((void*)1)
#define MPI_SUCCESS 0

int MPI_Init(int* argc, char*** argv);
int MPI_Finalize(void);
int MPI_Comm_rank(MPI_Comm comm, int* rank);
int MPI_Comm_size(MPI_Comm comm, int* size);
int MPI_Barrier(MPI_Comm comm);
int MPI_Allreduce(const void* src, void* dst, int count, MPI_Datatype t, MPI_Op op, MPI_Comm comm);
int MPI_Reduce(const void* src, void* dst, int count, MPI_Datatype t, MPI_Op op, int root, MPI_Comm comm);
int MPI_Bcast(void* buf, int count, MPI_Datatype t, int root, MPI_Comm comm);
int MPI_Scatter(const void* src, int scount, MPI_Datatype st, void* dst, int rcount, MPI_Datatype rt, int root, MPI_Comm comm);
int MPI_Gather(const void* src, int scount, MPI_Datatype st, void* dst, int rcount, MPI_Datatype rt, int root, MPI_Comm comm);
double MPI_Wtime(void);

#ifdef __cplusplus
}
#endif
#endif
