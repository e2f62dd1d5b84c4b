/*
 * Single-rank stand-in for the MPI API, used only to compile the reference
 * EU3D sources into the oracle library under oracle/_ref (test
 * infrastructure).  Every call behaves as MPI would on a communicator of size
 * one: reductions and gathers copy the send buffer, point-to-point calls are
 * only ever issued to MPI_PROC_NULL by a single rank, and waits return at once.
 */
#ifndef EU3D_ORACLE_MPI_STUB_H
#define EU3D_ORACLE_MPI_STUB_H

#include <string.h>
#include <time.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_INT 1
#define MPI_DOUBLE 2
#define MPI_MIN 10
#define MPI_MAX 11
#define MPI_SUM 12
#define MPI_PROC_NULL (-2)
#define MPI_REQUEST_NULL (-1)
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)

static inline size_t eu3d_stub_size(MPI_Datatype t) { return t == MPI_DOUBLE ? sizeof(double) : sizeof(int); }

static inline int MPI_Init(int *, char ***) { return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm, int *n) { *n = 1; return 0; }
static inline double MPI_Wtime(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return 0; }
static inline int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm)
{
    memcpy(r, s, (size_t)n * eu3d_stub_size(t));
    return 0;
}
static inline int MPI_Allgather(const void *s, int n, MPI_Datatype t, void *r, int, MPI_Datatype, MPI_Comm)
{
    memcpy(r, s, (size_t)n * eu3d_stub_size(t));
    return 0;
}
static inline int MPI_Gather(const void *s, int n, MPI_Datatype t, void *r, int, MPI_Datatype, int, MPI_Comm)
{
    memcpy(r, s, (size_t)n * eu3d_stub_size(t));
    return 0;
}
static inline int MPI_Isend(const void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *q)
{
    *q = MPI_REQUEST_NULL;
    return 0;
}
static inline int MPI_Irecv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *q)
{
    *q = MPI_REQUEST_NULL;
    return 0;
}
static inline int MPI_Recv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status *) { return 0; }
static inline int MPI_Waitall(int, MPI_Request *, MPI_Status *) { return 0; }

#endif
