/*
 * Single-rank MPI stand-in used ONLY to compile the reference's own C sources
 * into the test oracle (oracle/_ref).  Test infrastructure, never shipped.
 *
 * With one rank every point-to-point exchange in the reference is a
 * self-exchange of a buffer it has just filled (matcopy_elastic.c:76-81,
 * exchange_v.c:100-101), so a no-op send/receive leaves exactly the values the
 * real MPI library would deliver.  Reductions over one rank copy through.
 */
#ifndef IFOS_ORACLE_MPI_STUB_H
#define IFOS_ORACLE_MPI_STUB_H

#include <string.h>
#include <stdlib.h>
#include <time.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_FLOAT 4
#define MPI_DOUBLE 8
#define MPI_INT 4
#define MPI_CHAR 1
#define MPI_SUM 0
#define MPI_MAX 1
#define MPI_MIN 2
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_BSEND_OVERHEAD 0
#define MPI_IN_PLACE ((void *)1)

static inline double MPI_Wtime(void) { return (double)clock() / (double)CLOCKS_PER_SEC; }
static inline int MPI_Abort(MPI_Comm c, int code) { (void)c; exit(code); return 0; }
static inline int MPI_Barrier(MPI_Comm c) { (void)c; return 0; }
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
static inline int MPI_Allreduce(const void *in, void *out, int n, MPI_Datatype t, MPI_Op op, MPI_Comm c) {
    (void)op; (void)c;
    if (in != MPI_IN_PLACE && in != out) memcpy(out, in, (size_t)n * (size_t)t);
    return 0;
}
static inline int MPI_Bcast(void *b, int n, MPI_Datatype t, int r, MPI_Comm c) {
    (void)b; (void)n; (void)t; (void)r; (void)c; return 0;
}
static inline int MPI_Comm_rank(MPI_Comm c, int *r) { (void)c; *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm c, int *s) { (void)c; *s = 1; return 0; }
/* the rest of what the whole driver calls (src/IFOS2D.c, src/comm_ini.c):
 * start-up and shut-down, a split of the one-rank world into itself, the
 * persistent halo requests (never started with one rank) and the buffer of
 * the buffered sends */
static inline int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Comm_split(MPI_Comm c, int color, int key, MPI_Comm *out) {
    (void)c; (void)color; (void)key; *out = 0; return 0;
}
static inline int MPI_Bsend_init(const void *b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c, MPI_Request *r) {
    (void)b; (void)n; (void)t; (void)d; (void)tag; (void)c; *r = 0; return 0;
}
static inline int MPI_Recv_init(void *b, int n, MPI_Datatype t, int s, int tag, MPI_Comm c, MPI_Request *r) {
    (void)b; (void)n; (void)t; (void)s; (void)tag; (void)c; *r = 0; return 0;
}
static inline int MPI_Buffer_attach(void *b, int n) { (void)b; (void)n; return 0; }
static inline int MPI_Buffer_detach(void *b, int *n) { (void)b; (void)n; return 0; }

#endif
