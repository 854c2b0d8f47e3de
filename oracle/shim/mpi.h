/*
 * oracle/shim/mpi.h -- single-rank stand-in for the MPI subset the reference
 * solver calls (Solver/src/solver.c, force.c, sys_msr.c).  Test infrastructure
 * only: it lets the reference's own sources compile and run as one rank in a
 * container that has no MPI.  With one rank every collective is a copy (or a
 * no-op for MPI_IN_PLACE).  A datatype is represented by its size in bytes.
 */
#ifndef NS2D_SHIM_MPI_H
#define NS2D_SHIM_MPI_H
#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;

#define MPI_COMM_WORLD 0
#define MPI_IN_PLACE ((void*)1)
#define MPI_DOUBLE 8
#define MPI_INT 4
#define MPI_LONG 8
#define MPI_C_DOUBLE_COMPLEX 16
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_SUCCESS 0

static inline int MPI_Init(int* argc, char*** argv) { (void)argc; (void)argv; return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Comm_size(MPI_Comm c, int* s) { (void)c; *s = 1; return 0; }
static inline int MPI_Comm_rank(MPI_Comm c, int* r) { (void)c; *r = 0; return 0; }
static inline int MPI_Barrier(MPI_Comm c) { (void)c; return 0; }
static inline int MPI_Allreduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op op, MPI_Comm c) {
    (void)op; (void)c;
    if (s != MPI_IN_PLACE && n > 0) memmove(r, s, (size_t)n * (size_t)t);
    return 0;
}
static inline int MPI_Reduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op op, int root, MPI_Comm c) {
    (void)op; (void)root; (void)c;
    if (s != MPI_IN_PLACE && r && n > 0) memmove(r, s, (size_t)n * (size_t)t);
    return 0;
}
static inline int MPI_Allgather(const void* s, int sn, MPI_Datatype st, void* r, int rn, MPI_Datatype rt, MPI_Comm c) {
    (void)rn; (void)rt; (void)c;
    if (s != MPI_IN_PLACE && sn > 0) memmove(r, s, (size_t)sn * (size_t)st);
    return 0;
}
static inline int MPI_Gather(const void* s, int sn, MPI_Datatype st, void* r, int rn, MPI_Datatype rt, int root, MPI_Comm c) {
    (void)rn; (void)rt; (void)root; (void)c;
    if (s != MPI_IN_PLACE && r && sn > 0) memmove(r, s, (size_t)sn * (size_t)st);
    return 0;
}
static inline int MPI_Scatter(const void* s, int sn, MPI_Datatype st, void* r, int rn, MPI_Datatype rt, int root, MPI_Comm c) {
    (void)sn; (void)st; (void)root; (void)c;
    if (r != MPI_IN_PLACE && rn > 0) memmove(r, s, (size_t)rn * (size_t)rt);
    return 0;
}
static inline int MPI_Bcast(void* b, int n, MPI_Datatype t, int root, MPI_Comm c) {
    (void)b; (void)n; (void)t; (void)root; (void)c; return 0;
}
#endif
