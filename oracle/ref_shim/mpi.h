/*
 * Single-rank stand-in for the MPI subset the reference hot path calls
 * (TEST INFRASTRUCTURE ONLY: used to compile the unmodified reference sources
 * into oracle/_ref/ for pinning the oracle and for the CPU baseline).
 *
 * Semantics on one rank:
 *   - MPI_Cart_create records the periodic flags; MPI_Cart_shift returns the
 *     rank itself along a periodic dimension and MPI_PROC_NULL otherwise.
 *   - MPI_Type_indexed records (displacement, length) blocks in doubles.
 *   - MPI_Sendrecv to self gathers the send slice, then scatters it into the
 *     receive slice; with MPI_PROC_NULL it does nothing.
 *   - MPI_Allreduce copies (the reduction over one rank).
 *   The periodic flags live in one C++ inline function (external linkage), so
 *   every translation unit sees the flags MPI_Cart_create recorded.
 */
#ifndef NS_REF_SHIM_MPI_H
#define NS_REF_SHIM_MPI_H

#include <stdlib.h>
#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Info;
typedef int MPI_Op;
typedef struct { int dummy; } MPI_Status;
typedef struct ns_shim_type {
    int count;
    int* lens;
    int* disp;
    int elem;
}* MPI_Datatype;

#define MPI_COMM_WORLD 0
#define MPI_INFO_NULL 0
#define MPI_PROC_NULL (-2)
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_MIN 1
#define MPI_DOUBLE (ns_shim_double_type())

inline MPI_Datatype ns_shim_double_type(void) {
    static struct ns_shim_type t = {0, 0, 0, 1};
    return &t;
}

inline int* ns_shim_periods(void) {
    static int p[3] = {0, 0, 0};
    return p;
}

static inline int MPI_Init(int*, char***) { return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return 0; }
static inline int MPI_Cart_create(MPI_Comm, int ndims, const int*, const int* periods, int,
                                  MPI_Comm* out) {
    for (int d = 0; d < ndims && d < 3; d++) ns_shim_periods()[d] = periods[d];
    *out = 0;
    return 0;
}
static inline int MPI_Cart_coords(MPI_Comm, int, int maxdims, int* coords) {
    for (int d = 0; d < maxdims; d++) coords[d] = 0;
    return 0;
}
static inline int MPI_Cart_shift(MPI_Comm, int dim, int, int* src, int* dst) {
    int r = ns_shim_periods()[dim] ? 0 : MPI_PROC_NULL;
    *src = r;
    *dst = r;
    return 0;
}
static inline int MPI_Type_indexed(int count, const int* lens, const int* disp, MPI_Datatype,
                                   MPI_Datatype* out) {
    MPI_Datatype t = (MPI_Datatype)malloc(sizeof(struct ns_shim_type));
    t->count = count;
    t->elem = 0;
    t->lens = (int*)malloc(sizeof(int) * (count > 0 ? count : 1));
    t->disp = (int*)malloc(sizeof(int) * (count > 0 ? count : 1));
    for (int b = 0; b < count; b++) {
        t->lens[b] = lens[b];
        t->disp[b] = disp[b];
    }
    *out = t;
    return 0;
}
static inline int MPI_Type_commit(MPI_Datatype*) { return 0; }
static inline int MPI_Type_free(MPI_Datatype* t) {
    if (t && *t && !(*t)->elem) {
        free((*t)->lens);
        free((*t)->disp);
        free(*t);
    }
    *t = 0;
    return 0;
}
static inline int MPI_Sendrecv(const void* sbuf, int, MPI_Datatype st, int dest, int, void* rbuf,
                               int, MPI_Datatype rt, int source, int, MPI_Comm, MPI_Status*) {
    if (dest == MPI_PROC_NULL || source == MPI_PROC_NULL) return 0;
    size_t total = 0;
    for (int b = 0; b < st->count; b++) total += (size_t)st->lens[b];
    double* tmp = (double*)malloc(sizeof(double) * (total ? total : 1));
    const double* s = (const double*)sbuf;
    double* r = (double*)rbuf;
    size_t c = 0;
    for (int b = 0; b < st->count; b++)
        for (int e = 0; e < st->lens[b]; e++) tmp[c++] = s[st->disp[b] + e];
    c = 0;
    for (int b = 0; b < rt->count; b++)
        for (int e = 0; e < rt->lens[b]; e++) r[rt->disp[b] + e] = tmp[c++];
    free(tmp);
    return 0;
}
static inline int MPI_Allreduce(const void* s, void* r, int count, MPI_Datatype, MPI_Op,
                                MPI_Comm) {
    memcpy(r, s, sizeof(double) * (size_t)count);
    return 0;
}

#endif
