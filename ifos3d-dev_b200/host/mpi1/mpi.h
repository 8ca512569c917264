/*
 * One-rank MPI for the reference's host C code where no MPI library is
 * installed: the drop-in host (ifos3d-dev_b200/host, the reference's ifos3d.c
 * driving the B200 engine on one rank) and the CPU builds of the reference
 * that the tests compare against.
 *
 * Semantics are those of a real one-rank MPI run:
 *  - point-to-point calls are no-ops that leave the receive buffer untouched,
 *    exactly like MPI_Recv/Sendrecv_replace from MPI_PROC_NULL (this is what
 *    makes matcopy.c wrap the model ghost layers periodically on one rank);
 *  - Allreduce copies send -> recv (sum over one rank), Bcast/Barrier are no-ops;
 *  - MPI_Wtime is clock_gettime(CLOCK_MONOTONIC).
 */
#ifndef IFOSB_ONE_RANK_MPI_H
#define IFOSB_ONE_RANK_MPI_H

#include <string.h>
#include <stdlib.h>
#include <stdio.h>
#include <time.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_FLOAT 1
#define MPI_INT 2
#define MPI_CHAR 3
#define MPI_DOUBLE 4
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_PROC_NULL (-1)
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)
#define MPI_SUCCESS 0

static inline size_t ifos_stub_tsize(MPI_Datatype t) {
    switch (t) {
    case MPI_FLOAT: return sizeof(float);
    case MPI_INT: return sizeof(int);
    case MPI_CHAR: return 1;
    case MPI_DOUBLE: return sizeof(double);
    default: return 1;
    }
}

static inline int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Comm_size(MPI_Comm c, int *n) { (void)c; *n = 1; return 0; }
static inline int MPI_Comm_rank(MPI_Comm c, int *r) { (void)c; *r = 0; return 0; }
static inline int MPI_Barrier(MPI_Comm c) { (void)c; return 0; }
static inline int MPI_Abort(MPI_Comm c, int code) { (void)c; fprintf(stderr, "MPI_Abort(%d)\n", code); exit(code ? code : 1); }
static inline double MPI_Wtime(void) {
    struct timespec ts; clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}
static inline int MPI_Bcast(void *b, int n, MPI_Datatype t, int root, MPI_Comm c) {
    (void)b; (void)n; (void)t; (void)root; (void)c; return 0;
}
static inline int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, MPI_Comm c) {
    (void)op; (void)c;
    if (s != r) memmove(r, s, (size_t)n * ifos_stub_tsize(t));
    return 0;
}
static inline int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, int root, MPI_Comm c) {
    (void)root; return MPI_Allreduce(s, r, n, t, op, c);
}
static inline int MPI_Send(const void *b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c) {
    (void)b; (void)n; (void)t; (void)d; (void)tag; (void)c; return 0;
}
static inline int MPI_Bsend(const void *b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c) {
    (void)b; (void)n; (void)t; (void)d; (void)tag; (void)c; return 0;
}
static inline int MPI_Recv(void *b, int n, MPI_Datatype t, int s, int tag, MPI_Comm c, MPI_Status *st) {
    (void)b; (void)n; (void)t; (void)s; (void)tag; (void)c; (void)st; return 0;
}
static inline int MPI_Sendrecv_replace(void *b, int n, MPI_Datatype t, int d, int st, int s, int rt,
                                       MPI_Comm c, MPI_Status *status) {
    (void)b; (void)n; (void)t; (void)d; (void)st; (void)s; (void)rt; (void)c; (void)status; return 0;
}
static inline int MPI_Bsend_init(const void *b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c, MPI_Request *r) {
    (void)b; (void)n; (void)t; (void)d; (void)tag; (void)c; *r = 0; return 0;
}
static inline int MPI_Recv_init(void *b, int n, MPI_Datatype t, int s, int tag, MPI_Comm c, MPI_Request *r) {
    (void)b; (void)n; (void)t; (void)s; (void)tag; (void)c; *r = 0; return 0;
}
static inline int MPI_Start(MPI_Request *r) { (void)r; return 0; }
static inline int MPI_Wait(MPI_Request *r, MPI_Status *s) { (void)r; (void)s; return 0; }
static inline int MPI_Waitall(int n, MPI_Request *r, MPI_Status *s) { (void)n; (void)r; (void)s; return 0; }
static inline int MPI_Request_free(MPI_Request *r) { (void)r; return 0; }
static inline int MPI_Buffer_attach(void *b, int n) { (void)b; (void)n; return 0; }
static inline int MPI_Buffer_detach(void *b, int *n) { (void)b; (void)n; return 0; }

#endif
