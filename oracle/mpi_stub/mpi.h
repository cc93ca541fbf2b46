/* Single-rank MPI stand-in used only to compile the reference's level-set
 * sources into the CPU oracle (oracle/_ref).  Every collective is the
 * identity on one rank; point-to-point calls are never reached because the
 * reference switches communication off when the world has one rank
 * (src/ghostcell.cpp:38-39).  This header is test infrastructure: it is not
 * part of the shipped library. */
#ifndef R3D_ORACLE_MPI_STUB_H
#define R3D_ORACLE_MPI_STUB_H

#include <string.h>
#include <time.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef long MPI_Aint;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 1
#define MPI_COMM_NULL 0
#define MPI_REQUEST_NULL 0
#define MPI_PROC_NULL (-2)
#define MPI_BOTTOM ((void*)0)
#define MPI_CART_TOPOLOGY 2
#define MPI_INT 1
#define MPI_DOUBLE 2
#define MPI_SUM 1
#define MPI_MIN 2
#define MPI_MAX 3
#define MPI_STATUS_IGNORE ((MPI_Status*)0)

static inline size_t r3d_mpi_size(MPI_Datatype t) { return t == MPI_DOUBLE ? sizeof(double) : sizeof(int); }

static inline int MPI_Init(int*, char***) { return 0; }
static inline int MPI_Finalize() { return 0; }
static inline int MPI_Comm_dup(MPI_Comm c, MPI_Comm* o) { *o = c; return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return 0; }
static inline int MPI_Comm_free(MPI_Comm* c) { *c = MPI_COMM_NULL; return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline double MPI_Wtime() {
    struct timespec ts; clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}
static inline int MPI_Allreduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
    if (s != r) memmove(r, s, (size_t)n * r3d_mpi_size(t)); return 0;
}
static inline int MPI_Reduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
    if (s != r) memmove(r, s, (size_t)n * r3d_mpi_size(t)); return 0;
}
static inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return 0; }
static inline int MPI_Gather(const void* s, int n, MPI_Datatype t, void* r, int, MPI_Datatype, int, MPI_Comm) {
    if (s != r) memmove(r, s, (size_t)n * r3d_mpi_size(t)); return 0;
}
static inline int MPI_Allgather(const void* s, int n, MPI_Datatype t, void* r, int, MPI_Datatype, MPI_Comm) {
    if (s != r) memmove(r, s, (size_t)n * r3d_mpi_size(t)); return 0;
}
static inline int MPI_Gatherv(const void* s, int n, MPI_Datatype t, void* r, const int*, const int* d, MPI_Datatype, int, MPI_Comm) {
    memmove((char*)r + (size_t)d[0] * r3d_mpi_size(t), s, (size_t)n * r3d_mpi_size(t)); return 0;
}
static inline int MPI_Allgatherv(const void* s, int n, MPI_Datatype t, void* r, const int*, const int* d, MPI_Datatype, MPI_Comm) {
    memmove((char*)r + (size_t)d[0] * r3d_mpi_size(t), s, (size_t)n * r3d_mpi_size(t)); return 0;
}
static inline int MPI_Isend(const void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request* q) { *q = 0; return 0; }
static inline int MPI_Irecv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request* q) { *q = 0; return 0; }
static inline int MPI_Wait(MPI_Request*, MPI_Status*) { return 0; }
static inline int MPI_Get_address(const void* p, MPI_Aint* a) { *a = (MPI_Aint)p; return 0; }
static inline int MPI_Dims_create(int, int n, int* d) { for (int i = 0; i < n; ++i) if (d[i] == 0) d[i] = 1; return 0; }
static inline int MPI_Cart_create(MPI_Comm c, int, const int*, const int*, int, MPI_Comm* o) { *o = c; return 0; }
static inline int MPI_Cart_shift(MPI_Comm, int, int, int* a, int* b) { *a = MPI_PROC_NULL; *b = MPI_PROC_NULL; return 0; }
static inline int MPI_Neighbor_alltoallw(const void*, const int*, const MPI_Aint*, const MPI_Datatype*,
                                         void*, const int*, const MPI_Aint*, const MPI_Datatype*, MPI_Comm) { return 0; }

#endif
