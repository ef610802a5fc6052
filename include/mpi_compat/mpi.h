/*
 * Single-process <mpi.h> for building paratt drivers against libparatt_b200
 * without an MPI installation.  One rank (rank 0, size 1); collectives are
 * copies, point-to-point calls report an error.  Use a real MPI's header
 * instead when one is installed.
 */
#ifndef PARATT_MPI_COMPAT_H
#define PARATT_MPI_COMPAT_H

#include <stdlib.h>
#include <string.h>
#include <time.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 1
#define MPI_INT 4
#define MPI_DOUBLE 8
#define MPI_SUM 1
#define MPI_SUCCESS 0
#define MPI_ERR_OTHER 15
#define MPI_IN_PLACE ((void*)1)

static inline int MPI_Init(int* argc, char*** argv) { (void)argc; (void)argv; return MPI_SUCCESS; }
static inline int MPI_Finalize(void) { return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm c, int* r) { (void)c; *r = 0; return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm c, int* s) { (void)c; *s = 1; return MPI_SUCCESS; }
static inline int MPI_Barrier(MPI_Comm c) { (void)c; return MPI_SUCCESS; }
static inline int MPI_Bcast(void* b, int n, MPI_Datatype t, int root, MPI_Comm c)
{ (void)b; (void)n; (void)t; (void)root; (void)c; return MPI_SUCCESS; }
static inline int MPI_Allreduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op op, MPI_Comm c)
{
    (void)op; (void)c;
    if (s != MPI_IN_PLACE) memcpy(r, s, (size_t)n * (size_t)t);
    return MPI_SUCCESS;
}
static inline int MPI_Abort(MPI_Comm c, int code) { (void)c; exit(code ? code : 1); return code; }
static inline double MPI_Wtime(void)
{ struct timespec ts; clock_gettime(CLOCK_MONOTONIC, &ts); return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec; }
static inline int MPI_Wait(MPI_Request* q, MPI_Status* s) { (void)q; (void)s; return MPI_SUCCESS; }

#endif
