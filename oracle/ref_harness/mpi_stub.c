/*
 * Single-rank definitions for the MPI calls that SHOCK's hot-path
 * translation units reference.  The harness runs one block per process
 * with no interfaces, so the point-to-point calls must never be reached;
 * they abort loudly if they are.  Collectives degenerate to copies.
 * Test infrastructure for the reference build under oracle/_ref.
 */
#include "mpi.h"
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

static size_t dtype_size(MPI_Datatype t)
{
    switch (t) {
    case MPI_FLOAT: return sizeof(float);
    case MPI_DOUBLE: return sizeof(double);
    case MPI_LONG_DOUBLE: return sizeof(long double);
    case MPI_INT: return sizeof(int);
    case MPI_CHAR: return 1;
    default: return 0;
    }
}

static void unreachable(const char *name)
{
    fprintf(stderr, "oracle/_ref: %s called in a single-block harness\n", name);
    abort();
}

int MPI_Init(int *a, char ***b) { (void)a; (void)b; return 0; }
int MPI_Finalize(void) { return 0; }
int MPI_Comm_size(MPI_Comm c, int *n) { (void)c; *n = 1; return 0; }
int MPI_Comm_rank(MPI_Comm c, int *r) { (void)c; *r = 0; return 0; }
int MPI_Barrier(MPI_Comm c) { (void)c; return 0; }
double MPI_Wtime(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}
int MPI_Abort(MPI_Comm c, int code) { (void)c; fprintf(stderr, "MPI_Abort(%d)\n", code); abort(); }
int MPI_Comm_get_attr(MPI_Comm c, int key, void *val, int *flag)
{
    static int tag_ub = 32767;
    static int *p = &tag_ub;
    (void)c; (void)key;
    *(int **)val = p;
    *flag = 1;
    return 0;
}
int MPI_Isend(const void *b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c, MPI_Request *r)
{ (void)b; (void)n; (void)t; (void)d; (void)tag; (void)c; (void)r; unreachable("MPI_Isend"); return 1; }
int MPI_Irecv(void *b, int n, MPI_Datatype t, int s, int tag, MPI_Comm c, MPI_Request *r)
{ (void)b; (void)n; (void)t; (void)s; (void)tag; (void)c; (void)r; unreachable("MPI_Irecv"); return 1; }
int MPI_Test(MPI_Request *r, int *f, MPI_Status *s) { (void)r; (void)s; *f = 1; return 0; }
int MPI_Waitall(int n, MPI_Request *r, MPI_Status *s) { (void)n; (void)r; (void)s; return 0; }
int MPI_Sendrecv(const void *a, int b, MPI_Datatype c, int d, int e, void *f, int g,
                 MPI_Datatype h, int i, int j, MPI_Comm k, MPI_Status *l)
{
    (void)a; (void)b; (void)c; (void)d; (void)e; (void)f; (void)g; (void)h;
    (void)i; (void)j; (void)k; (void)l;
    unreachable("MPI_Sendrecv");
    return 1;
}
int MPI_Allgather(const void *sb, int sn, MPI_Datatype st, void *rb, int rn, MPI_Datatype rt, MPI_Comm c)
{
    (void)rn; (void)rt; (void)c;
    memcpy(rb, sb, (size_t)sn * dtype_size(st));
    return 0;
}
int MPI_Reduce(const void *sb, void *rb, int n, MPI_Datatype t, MPI_Op op, int root, MPI_Comm c)
{
    (void)op; (void)root; (void)c;
    memcpy(rb, sb, (size_t)n * dtype_size(t));
    return 0;
}
int MPI_Bcast(void *b, int n, MPI_Datatype t, int root, MPI_Comm c)
{ (void)b; (void)n; (void)t; (void)root; (void)c; return 0; }
int MPI_Cart_create(MPI_Comm a, int b, const int *c, const int *d, int e, MPI_Comm *f)
{ (void)a; (void)b; (void)c; (void)d; (void)e; *f = 0; return 0; }
int MPI_Cart_coords(MPI_Comm a, int b, int c, int *d) { (void)a; (void)b; for (int i = 0; i < c; i++) d[i] = 0; return 0; }
int MPI_Cart_shift(MPI_Comm a, int b, int c, int *d, int *e) { (void)a; (void)b; (void)c; *d = *e = MPI_PROC_NULL; return 0; }
int MPI_Type_create_subarray(int a, const int *b, const int *c, const int *d, int e, MPI_Datatype f, MPI_Datatype *g)
{ (void)a; (void)b; (void)c; (void)d; (void)e; *g = f; return 0; }
int MPI_Type_commit(MPI_Datatype *t) { (void)t; return 0; }
int MPI_Type_size(MPI_Datatype t, int *s) { *s = (int)dtype_size(t); return 0; }
