/* Single-rank stand-in for the MPI API the reference's GPU sources reference (test
 * infrastructure: lets the reference's own kernels and host orchestration be compiled and run on
 * one GPU without an MPI installation).  One process, rank 0 of 1: reductions copy their input,
 * barriers return at once. */
#ifndef IB_REF_SHIM_MPI_H
#define IB_REF_SHIM_MPI_H

#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Fint;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;
typedef int MPI_Request;

#define MPI_COMM_WORLD 0
#define MPI_COMM_NULL (-1)
#define MPI_SUCCESS 0
#define MPI_DOUBLE 1
#define MPI_INT 2
#define MPI_INTEGER 3
#define MPI_FLOAT 4
#define MPI_LONG 5
#define MPI_BYTE 6
#define MPI_CHAR 7
#define MPI_SUM 1
#define MPI_PROD 2
#define MPI_MAX 3
#define MPI_MIN 4
#define MPI_LAND 5
#define MPI_LOR 6
#define MPI_STATUS_IGNORE ((MPI_Status *)0)

static inline int ib_shim_size(MPI_Datatype t)
{
    switch (t) {
    case MPI_DOUBLE: return 8;
    case MPI_LONG: return 8;
    case MPI_BYTE: case MPI_CHAR: return 1;
    default: return 4;
    }
}
static inline int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op o, MPI_Comm c)
{
    (void)o; (void)c;
    if (s != r) memcpy(r, s, (size_t)n * ib_shim_size(t));
    return MPI_SUCCESS;
}
static inline int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op o, int root, MPI_Comm c)
{
    (void)root;
    return MPI_Allreduce(s, r, n, t, o, c);
}
static inline int MPI_Bcast(void *b, int n, MPI_Datatype t, int root, MPI_Comm c) { (void)b; (void)n; (void)t; (void)root; (void)c; return MPI_SUCCESS; }
static inline int MPI_Barrier(MPI_Comm c) { (void)c; return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm c, int *r) { (void)c; *r = 0; return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm c, int *s) { (void)c; *s = 1; return MPI_SUCCESS; }
static inline MPI_Comm MPI_Comm_f2c(MPI_Fint f) { return (MPI_Comm)f; }
static inline MPI_Fint MPI_Comm_c2f(MPI_Comm c) { return (MPI_Fint)c; }
static inline int MPI_Abort(MPI_Comm c, int e) { (void)c; (void)e; return MPI_SUCCESS; }
static inline int MPI_Initialized(int *f) { *f = 1; return MPI_SUCCESS; }
static inline int MPI_Comm_free(MPI_Comm *c) { (void)c; return MPI_SUCCESS; }
static inline int MPI_Comm_split(MPI_Comm c, int a, int b, MPI_Comm *n) { (void)a; (void)b; *n = c; return MPI_SUCCESS; }
static inline int MPI_Comm_dup(MPI_Comm c, MPI_Comm *n) { *n = c; return MPI_SUCCESS; }
static inline int MPI_Cart_create(MPI_Comm c, int nd, const int *d, const int *p, int re, MPI_Comm *n)
{ (void)nd; (void)d; (void)p; (void)re; *n = c; return MPI_SUCCESS; }
static inline int MPI_Cart_sub(MPI_Comm c, const int *r, MPI_Comm *n) { (void)r; *n = c; return MPI_SUCCESS; }
static inline int MPI_Allgather(const void *s, int sn, MPI_Datatype st, void *r, int rn, MPI_Datatype rt, MPI_Comm c)
{ (void)rn; (void)rt; (void)c; memcpy(r, s, (size_t)sn * ib_shim_size(st)); return MPI_SUCCESS; }
static inline int MPI_Isend(const void *b, int n, MPI_Datatype t, int d, int g, MPI_Comm c, MPI_Request *q)
{ (void)b; (void)n; (void)t; (void)d; (void)g; (void)c; *q = 0; return MPI_SUCCESS; }
static inline int MPI_Irecv(void *b, int n, MPI_Datatype t, int s, int g, MPI_Comm c, MPI_Request *q)
{ (void)b; (void)n; (void)t; (void)s; (void)g; (void)c; *q = 0; return MPI_SUCCESS; }
static inline int MPI_Waitall(int n, MPI_Request *q, MPI_Status *s) { (void)n; (void)q; (void)s; return MPI_SUCCESS; }
static inline int MPI_Send(const void *b, int n, MPI_Datatype t, int d, int g, MPI_Comm c)
{ (void)b; (void)n; (void)t; (void)d; (void)g; (void)c; return MPI_SUCCESS; }
static inline int MPI_Recv(void *b, int n, MPI_Datatype t, int s, int g, MPI_Comm c, MPI_Status *st)
{ (void)b; (void)n; (void)t; (void)s; (void)g; (void)c; (void)st; return MPI_SUCCESS; }

#endif
