/* Serial single-rank stand-in for the MPI API subset the reference calls.
 *
 * Test infrastructure only: lets the reference's own sources (tem.cpp and the
 * build/Makefile:28 object list) compile and run as one rank so they can serve
 * as the oracle.  Semantics are those of MPI with size 1 and rank 0:
 * broadcasts are no-ops, gathers/scatters/reductions copy send -> receive. */
#ifndef MSF_ORACLE_SHIM_MPI_H
#define MSF_ORACLE_SHIM_MPI_H
#include <stddef.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_THREAD_FUNNELED 1
#define MPI_IN_PLACE ((void*)1)

#define MPI_CHAR 1
#define MPI_UNSIGNED_CHAR 2
#define MPI_UNSIGNED_SHORT 3
#define MPI_INT 4
#define MPI_UNSIGNED 5
#define MPI_UNSIGNED_LONG 6
#define MPI_UNSIGNED_LONG_LONG 7
#define MPI_DOUBLE 8

#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3

#ifdef __cplusplus
extern "C" {
#endif
int MPI_Init(int* argc, char*** argv);
int MPI_Init_thread(int* argc, char*** argv, int required, int* provided);
int MPI_Finalize(void);
int MPI_Comm_rank(MPI_Comm comm, int* rank);
int MPI_Comm_size(MPI_Comm comm, int* size);
int MPI_Barrier(MPI_Comm comm);
int MPI_Bcast(void* buf, int count, MPI_Datatype t, int root, MPI_Comm comm);
int MPI_Allgather(const void* sb, int sc, MPI_Datatype st, void* rb, int rc,
                  MPI_Datatype rt, MPI_Comm comm);
int MPI_Allgatherv(const void* sb, int sc, MPI_Datatype st, void* rb,
                   const int* rcounts, const int* displs, MPI_Datatype rt,
                   MPI_Comm comm);
int MPI_Gather(const void* sb, int sc, MPI_Datatype st, void* rb, int rc,
               MPI_Datatype rt, int root, MPI_Comm comm);
int MPI_Gatherv(const void* sb, int sc, MPI_Datatype st, void* rb,
                const int* rcounts, const int* displs, MPI_Datatype rt,
                int root, MPI_Comm comm);
int MPI_Scatter(const void* sb, int sc, MPI_Datatype st, void* rb, int rc,
                MPI_Datatype rt, int root, MPI_Comm comm);
int MPI_Scatterv(const void* sb, const int* scounts, const int* displs,
                 MPI_Datatype st, void* rb, int rc, MPI_Datatype rt, int root,
                 MPI_Comm comm);
int MPI_Reduce(const void* sb, void* rb, int count, MPI_Datatype t, MPI_Op op,
               int root, MPI_Comm comm);
int MPI_Allreduce(const void* sb, void* rb, int count, MPI_Datatype t,
                  MPI_Op op, MPI_Comm comm);
double MPI_Wtime(void);
#ifdef __cplusplus
}
#endif
#endif
