/* Oracle test shim: a single-rank MPI for compiling the reference's hot-path and ensemble
 * driver sources in one process.  Collectives copy send buffers to receive buffers. */
#ifndef DMS_SHIM_MPI_H
#define DMS_SHIM_MPI_H
#include <stddef.h>
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;
#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_CHAR 1
#define MPI_BYTE 1
#define MPI_INT 4
#define MPI_UNSIGNED 5
#define MPI_DOUBLE 8
#define MPI_UNSIGNED_LONG 9
#define MPI_UNSIGNED_LONG_LONG 10
#define MPI_UINT64_T 11
#define MPI_LONG 12
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_IN_PLACE ((void*)1)
#define MPI_REQUEST_NULL 0
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_THREAD_SINGLE 0
#define MPI_THREAD_FUNNELED 1
#define MPI_THREAD_SERIALIZED 2
#define MPI_THREAD_MULTIPLE 3
#ifdef __cplusplus
extern "C" {
#endif
int MPI_Init(int*, char***);
int MPI_Init_thread(int*, char***, int, int*);
int MPI_Finalize(void);
int MPI_Comm_size(MPI_Comm, int*);
int MPI_Comm_rank(MPI_Comm, int*);
int MPI_Barrier(MPI_Comm);
int MPI_Query_thread(int*);
int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm);
int MPI_Allreduce(const void*, void*, int, MPI_Datatype, MPI_Op, MPI_Comm);
int MPI_Allgather(const void*, int, MPI_Datatype, void*, int, MPI_Datatype, MPI_Comm);
int MPI_Allgatherv(const void*, int, MPI_Datatype, void*, const int*, const int*, MPI_Datatype, MPI_Comm);
int MPI_Gather(const void*, int, MPI_Datatype, void*, int, MPI_Datatype, int, MPI_Comm);
int MPI_Gatherv(const void*, int, MPI_Datatype, void*, const int*, const int*, MPI_Datatype, int, MPI_Comm);
int MPI_Ibarrier(MPI_Comm, MPI_Request*);
int MPI_Test(MPI_Request*, int*, MPI_Status*);
int MPI_Wait(MPI_Request*, MPI_Status*);
#ifdef __cplusplus
}
#endif
#endif
