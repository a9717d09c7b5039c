/* Single-rank stand-in for the handful of MPI calls GiftBTE's CPU solver makes.
 *
 * Test infrastructure only: it lets oracle/Makefile compile the unmodified
 * reference sources into oracle/_ref/BTE_CPU on a machine without an MPI
 * installation. With one rank every collective the reference issues is a copy
 * of the send buffer into the receive buffer (Allreduce/Allgather/Allgatherv)
 * or a no-op (Barrier, Send/Recv of the loop counter to other ranks, which
 * never exist). Written for this project; it is not derived from any MPI
 * implementation. */
#ifndef GBTE_ORACLE_MPI_STUB_H
#define GBTE_ORACLE_MPI_STUB_H
#include <string.h>
#include <stddef.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
/* datatype handles encode the element size in bytes */
#define MPI_CHAR 1
#define MPI_UNSIGNED_CHAR 1
#define MPI_UNSIGNED_SHORT 2
#define MPI_INT 4
#define MPI_UNSIGNED 4
#define MPI_FLOAT 104
#define MPI_DOUBLE 8
#define MPI_LONG 108
#define MPI_UNSIGNED_LONG 208
#define MPI_UNSIGNED_LONG_LONG 308
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_IN_PLACE ((void *)1)

static inline size_t gbte_stub_size(MPI_Datatype t) {
    switch (t) {
    case MPI_FLOAT: return 4;
    case MPI_LONG: case MPI_UNSIGNED_LONG: case MPI_UNSIGNED_LONG_LONG: return 8;
    default: return (size_t)t;
    }
}
static inline int MPI_Init(int *, char ***) { return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Comm_size(MPI_Comm, int *n) { *n = 1; return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
    if (s != MPI_IN_PLACE && s != r) memmove(r, s, (size_t)n * gbte_stub_size(t));
    return 0;
}
static inline int MPI_Allgather(const void *s, int n, MPI_Datatype t, void *r, int, MPI_Datatype, MPI_Comm) {
    if (s != MPI_IN_PLACE && s != r) memmove(r, s, (size_t)n * gbte_stub_size(t));
    return 0;
}
static inline int MPI_Allgatherv(const void *s, int n, MPI_Datatype t, void *r, const int *, const int *displs,
                                 MPI_Datatype, MPI_Comm) {
    char *dst = (char *)r + (size_t)displs[0] * gbte_stub_size(t);
    if (s != MPI_IN_PLACE && s != dst) memmove(dst, s, (size_t)n * gbte_stub_size(t));
    return 0;
}
static inline int MPI_Send(const void *, int, MPI_Datatype, int, int, MPI_Comm) { return 0; }
static inline int MPI_Recv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status *) { return 0; }
#endif
