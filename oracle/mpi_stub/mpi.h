/*
 * Single-process stand-in for <mpi.h>, used only to compile the reference
 * paratt sources into the CPU oracle (oracle/_ref).  TEST INFRASTRUCTURE:
 * nothing in the product links against this header.
 *
 * World size is 1 and the rank is 0.  With one rank the reference's TSQR tree
 * has a single node (tsqr.c:274-402), so no point-to-point message is ever
 * posted on the rounding path; collectives reduce to copies.
 */
#ifndef PARATT_ORACLE_MPI_STUB_H
#define PARATT_ORACLE_MPI_STUB_H

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 1
#define MPI_DOUBLE 8
#define MPI_INT 4
#define MPI_SUM 1
#define MPI_SUCCESS 0
#define MPI_IN_PLACE ((void*)1)

static inline int mpistub_size(MPI_Datatype t) { return t == MPI_DOUBLE ? 8 : 4; }

static inline int MPI_Init(int* argc, char*** argv) { (void)argc; (void)argv; return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Comm_rank(MPI_Comm c, int* r) { (void)c; *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm c, int* s) { (void)c; *s = 1; return 0; }
static inline int MPI_Comm_dup(MPI_Comm c, MPI_Comm* out) { *out = c; return 0; }
static inline int MPI_Comm_free(MPI_Comm* c) { (void)c; return 0; }
static inline int MPI_Barrier(MPI_Comm c) { (void)c; return 0; }
static inline int MPI_Bcast(void* b, int n, MPI_Datatype t, int root, MPI_Comm c)
{ (void)b; (void)n; (void)t; (void)root; (void)c; return 0; }
static inline int MPI_Allreduce(const void* s, void* r, int n, MPI_Datatype t,
                                MPI_Op op, MPI_Comm c)
{
    (void)op; (void)c;
    if (s != MPI_IN_PLACE) memcpy(r, s, (size_t)n * (size_t)mpistub_size(t));
    return 0;
}
static inline int MPI_Abort(MPI_Comm c, int code)
{ (void)c; fprintf(stderr, "MPI_Abort(%d) in single-process stub\n", code); exit(code ? code : 1); }
/* Messages a rank sends to itself (the reference's ordered file writer,
 * paratt.c:1640-1688, passes a token to rank 0 when there is one rank) are
 * kept in a small per-translation-unit FIFO.  Any other destination aborts. */
static char mpistub_box[4096];
static size_t mpistub_head = 0, mpistub_tail = 0;
static inline int mpistub_p2p(const char* what)
{ fprintf(stderr, "%s: only self-messages exist with one rank\n", what); abort(); return 1; }
static inline int mpistub_put(const void* b, int n, MPI_Datatype t, int peer)
{
    size_t len = (size_t)n * (size_t)mpistub_size(t);
    if (peer != 0 || mpistub_tail + len > sizeof(mpistub_box)) return mpistub_p2p("MPI_Send");
    memcpy(mpistub_box + mpistub_tail, b, len);
    mpistub_tail += len;
    return 0;
}
static inline int mpistub_get(void* b, int n, MPI_Datatype t, int peer)
{
    size_t len = (size_t)n * (size_t)mpistub_size(t);
    if (peer != 0 || mpistub_head + len > mpistub_tail) return mpistub_p2p("MPI_Recv");
    memcpy(b, mpistub_box + mpistub_head, len);
    mpistub_head += len;
    if (mpistub_head == mpistub_tail) mpistub_head = mpistub_tail = 0;
    return 0;
}
static inline int MPI_Send(const void* b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c)
{ (void)tag; (void)c; return mpistub_put(b, n, t, d); }
static inline int MPI_Recv(void* b, int n, MPI_Datatype t, int s, int tag, MPI_Comm c, MPI_Status* st)
{ (void)tag; (void)c; (void)st; return mpistub_get(b, n, t, s); }
static inline int MPI_Isend(const void* b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c, MPI_Request* q)
{ (void)tag; (void)c; (void)q; return mpistub_put(b, n, t, d); }
static inline int MPI_Irecv(void* b, int n, MPI_Datatype t, int s, int tag, MPI_Comm c, MPI_Request* q)
{ (void)tag; (void)c; (void)q; return mpistub_get(b, n, t, s); }
static inline int MPI_Wait(MPI_Request* q, MPI_Status* st) { (void)q; (void)st; return 0; }
static inline double MPI_Wtime(void)
{ struct timespec ts; clock_gettime(CLOCK_MONOTONIC, &ts); return ts.tv_sec + 1e-9 * ts.tv_nsec; }

#endif
