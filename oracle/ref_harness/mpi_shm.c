/*
 * Multi-process stand-in for the MPI subset SHOCK's hot-path translation
 * units use, so that SHOCK's own halo exchange (TransferFlowParameterWithGhosts
 * and TransferMeshParameter, src/Functions.c:3481-3684) runs between ranks:
 * the ranks are processes forked by shm_run() that share one anonymous
 * mapping.  Test infrastructure for the reference build under oracle/_ref
 * (the multi-rank oracle of the blocks-on-one-GPU path) -- not MPI, and not
 * part of the shipped library.
 *
 *   point to point  buffered: MPI_Isend copies the message into a slot of
 *                   the (source, destination) mailbox and completes at once;
 *                   MPI_Irecv records the request, MPI_Test takes a full slot
 *                   with the matching tag (messages of one tag arrive in
 *                   order).  A rank's receives complete in the order it
 *                   posted them: MPI leaves that order open, and SHOCK
 *                   unpacks each interface as its receive completes, with
 *                   the ghost corners of neighbouring interfaces written by
 *                   both, so its results depend on the order.  Posting order
 *                   is the schedule in which every message has arrived before
 *                   the receiver polls, and makes the runs reproducible;
 *   collectives     Barrier (sense-reversing counter), Allgather, Reduce
 *                   (SUM, MAX), Bcast through a shared staging area;
 *   MPI-IO          read-only, independent: a file is a POSIX descriptor,
 *                   the view a byte displacement (what loadDivision,
 *                   src/Load.c:191-250, uses to read its rank's row);
 *   waits           every spin gives up after SHM_WAIT_S seconds and aborts
 *                   the whole job (a rank that never arrives is an error of
 *                   the test set-up, not something to wait out).
 */
#include "mpi.h"

#include <signal.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <sys/wait.h>
#include <time.h>
#include <unistd.h>

#define SHM_SLOTS 16          /* messages in flight per (source, destination) */
#define SHM_WAIT_S 120.0
#define SHM_STAGE_BYTES 4096  /* collective staging per rank */

typedef struct {
    volatile int full;
    int tag;
    size_t bytes;
    size_t seq;               /* arrival order among full slots */
} slot_t;

typedef struct {
    int nranks;
    size_t slot_bytes;
    volatile int bar_count, bar_sense;
    volatile int abort_code;
    size_t seq;
} shm_head_t;

static shm_head_t *g_head;
static char *g_base;          /* the whole mapping */
static size_t g_map_bytes;
static int g_rank, g_local_sense;

typedef struct {
    int used, src, tag, recv;
    void *buf;
    size_t bytes;
    size_t post;              /* posting order */
    int done;                 /* data received, not yet reported */
} req_t;

static size_t g_posted;

static req_t g_req[4096];

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

static double now_s(void)
{
    struct timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}

static slot_t *slot(int src, int dst, int s)
{
    char *p = g_base + sizeof(shm_head_t);
    size_t per = sizeof(slot_t) + g_head->slot_bytes;
    return (slot_t *)(p + (((size_t)src * g_head->nranks + dst) * SHM_SLOTS + s) * per);
}

static char *slot_data(slot_t *s) { return (char *)(s + 1); }

static char *stage(int r)
{
    size_t per = sizeof(slot_t) + g_head->slot_bytes;
    char *p = g_base + sizeof(shm_head_t) + (size_t)g_head->nranks * g_head->nranks * SHM_SLOTS * per;
    return p + (size_t)r * SHM_STAGE_BYTES;
}

static void check_wait(double t0, const char *what)
{
    if (g_head->abort_code) _exit(3);
    if (now_s() - t0 > SHM_WAIT_S) {
        fprintf(stderr, "mpi_shm: rank %d gave up waiting in %s\n", g_rank, what);
        g_head->abort_code = 1;
        _exit(3);
    }
}

int MPI_Init(int *a, char ***b) { (void)a; (void)b; return 0; }
int MPI_Finalize(void) { return 0; }
int MPI_Comm_size(MPI_Comm c, int *n) { (void)c; *n = g_head ? g_head->nranks : 1; return 0; }
int MPI_Comm_rank(MPI_Comm c, int *r) { (void)c; *r = g_rank; return 0; }

int MPI_Barrier(MPI_Comm c)
{
    (void)c;
    if (!g_head || g_head->nranks == 1) return 0;
    g_local_sense = !g_local_sense;
    if (__atomic_add_fetch(&g_head->bar_count, 1, __ATOMIC_ACQ_REL) == g_head->nranks) {
        __atomic_store_n(&g_head->bar_count, 0, __ATOMIC_RELAXED);
        __atomic_store_n(&g_head->bar_sense, g_local_sense, __ATOMIC_RELEASE);
    } else {
        const double t0 = now_s();
        while (__atomic_load_n(&g_head->bar_sense, __ATOMIC_ACQUIRE) != g_local_sense) check_wait(t0, "MPI_Barrier");
    }
    return 0;
}

double MPI_Wtime(void) { return now_s(); }

int MPI_Abort(MPI_Comm c, int code)
{
    (void)c;
    fprintf(stderr, "MPI_Abort(%d) on rank %d\n", code, g_rank);
    if (g_head) g_head->abort_code = code ? code : 1;
    _exit(2);
}

int MPI_Comm_get_attr(MPI_Comm c, int key, void *val, int *flag)
{
    static int tag_ub = 2147483647;
    (void)c; (void)key;
    *(int **)val = &tag_ub;
    *flag = 1;
    return 0;
}

int MPI_Isend(const void *b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c, MPI_Request *r)
{
    (void)c;
    const size_t bytes = (size_t)n * dtype_size(t);
    if (bytes > g_head->slot_bytes) {
        fprintf(stderr, "mpi_shm: message of %zu bytes exceeds the slot size\n", bytes);
        MPI_Abort(0, 4);
    }
    const double t0 = now_s();
    for (;;) {
        for (int s = 0; s < SHM_SLOTS; s++) {
            slot_t *sl = slot(g_rank, d, s);
            if (__atomic_load_n(&sl->full, __ATOMIC_ACQUIRE)) continue;
            memcpy(slot_data(sl), b, bytes);
            sl->tag = tag;
            sl->bytes = bytes;
            sl->seq = __atomic_add_fetch(&g_head->seq, 1, __ATOMIC_ACQ_REL);
            __atomic_store_n(&sl->full, 1, __ATOMIC_RELEASE);
            *r = MPI_REQUEST_NULL;   /* buffered: complete */
            return 0;
        }
        check_wait(t0, "MPI_Isend (mailbox full)");
    }
}

int MPI_Irecv(void *b, int n, MPI_Datatype t, int s, int tag, MPI_Comm c, MPI_Request *r)
{
    (void)c;
    for (int i = 1; i < 4096; i++)
        if (!g_req[i].used) {
            g_req[i] = (req_t){1, s, tag, 1, b, (size_t)n * dtype_size(t), ++g_posted, 0};
            *r = i;
            return 0;
        }
    fprintf(stderr, "mpi_shm: too many requests\n");
    MPI_Abort(0, 5);
    return 1;
}

/* Take the oldest full slot from src with tag into req; 1 if done. */
static int try_recv(req_t *q)
{
    slot_t *best = NULL;
    for (int s = 0; s < SHM_SLOTS; s++) {
        slot_t *sl = slot(q->src, g_rank, s);
        if (!__atomic_load_n(&sl->full, __ATOMIC_ACQUIRE) || sl->tag != q->tag) continue;
        if (!best || sl->seq < best->seq) best = sl;
    }
    if (!best) return 0;
    if (best->bytes != q->bytes) {
        fprintf(stderr, "mpi_shm: rank %d expected %zu bytes from %d, got %zu\n", g_rank, q->bytes, q->src,
                best->bytes);
        MPI_Abort(0, 6);
    }
    memcpy(q->buf, slot_data(best), q->bytes);
    __atomic_store_n(&best->full, 0, __ATOMIC_RELEASE);
    return 1;
}

int MPI_Test(MPI_Request *r, int *f, MPI_Status *st)
{
    (void)st;
    if (*r == MPI_REQUEST_NULL) { *f = 1; return 0; }
    req_t *q = &g_req[*r];
    /* complete the pending receives posted up to this one, oldest first */
    for (;;) {
        req_t *old = NULL;
        for (int i = 1; i < 4096; i++) {
            req_t *c = &g_req[i];
            if (c->used && c->recv && !c->done && c->post <= q->post && (!old || c->post < old->post)) old = c;
        }
        if (!old || !try_recv(old)) break;
        old->done = 1;
    }
    *f = q->done;
    if (*f) { q->used = 0; *r = MPI_REQUEST_NULL; }
    return 0;
}

int MPI_Waitall(int n, MPI_Request *r, MPI_Status *st)
{
    (void)st;
    for (int i = 0; i < n; i++) {
        const double t0 = now_s();
        int f = 0;
        while (MPI_Test(&r[i], &f, NULL), !f) check_wait(t0, "MPI_Waitall");
    }
    return 0;
}

int MPI_Sendrecv(const void *a, int b, MPI_Datatype c, int d, int e, void *f, int g, MPI_Datatype h, int i, int j,
                 MPI_Comm k, MPI_Status *l)
{
    MPI_Request s, r;
    MPI_Isend(a, b, c, d, e, k, &s);
    MPI_Irecv(f, g, h, i, j, k, &r);
    return MPI_Waitall(1, &r, l);
}

int MPI_Allgather(const void *sb, int sn, MPI_Datatype st, void *rb, int rn, MPI_Datatype rt, MPI_Comm c)
{
    (void)rt; (void)rn;
    const size_t bytes = (size_t)sn * dtype_size(st);
    if (bytes > SHM_STAGE_BYTES) MPI_Abort(0, 7);
    MPI_Barrier(c);
    memcpy(stage(g_rank), sb, bytes);
    MPI_Barrier(c);
    for (int r = 0; r < g_head->nranks; r++) memcpy((char *)rb + r * bytes, stage(r), bytes);
    MPI_Barrier(c);
    return 0;
}

int MPI_Reduce(const void *sb, void *rb, int n, MPI_Datatype t, MPI_Op op, int root, MPI_Comm c)
{
    const size_t bytes = (size_t)n * dtype_size(t);
    if (bytes > SHM_STAGE_BYTES) MPI_Abort(0, 8);
    MPI_Barrier(c);
    memcpy(stage(g_rank), sb, bytes);
    MPI_Barrier(c);
    if (g_rank == root) {
        memcpy(rb, stage(0), bytes);
        for (int r = 1; r < g_head->nranks; r++)
            for (int i = 0; i < n; i++) {
                if (t == MPI_DOUBLE) {
                    double *o = (double *)rb + i, v = ((double *)stage(r))[i];
                    *o = op == MPI_MAX ? (v > *o ? v : *o) : *o + v;
                } else if (t == MPI_INT) {
                    int *o = (int *)rb + i, v = ((int *)stage(r))[i];
                    *o = op == MPI_MAX ? (v > *o ? v : *o) : *o + v;
                } else if (t == MPI_FLOAT) {
                    float *o = (float *)rb + i, v = ((float *)stage(r))[i];
                    *o = op == MPI_MAX ? (v > *o ? v : *o) : *o + v;
                } else {
                    long double *o = (long double *)rb + i, v = ((long double *)stage(r))[i];
                    *o = op == MPI_MAX ? (v > *o ? v : *o) : *o + v;
                }
            }
    }
    MPI_Barrier(c);
    return 0;
}

int MPI_Bcast(void *b, int n, MPI_Datatype t, int root, MPI_Comm c)
{
    const size_t bytes = (size_t)n * dtype_size(t);
    if (bytes > SHM_STAGE_BYTES) MPI_Abort(0, 9);
    MPI_Barrier(c);
    if (g_rank == root) memcpy(stage(root), b, bytes);
    MPI_Barrier(c);
    if (g_rank != root) memcpy(b, stage(root), bytes);
    MPI_Barrier(c);
    return 0;
}

int MPI_Cart_create(MPI_Comm a, int b, const int *c, const int *d, int e, MPI_Comm *f)
{ (void)a; (void)b; (void)c; (void)d; (void)e; *f = 0; return 0; }
int MPI_Cart_coords(MPI_Comm a, int b, int c, int *d) { (void)a; (void)b; for (int i = 0; i < c; i++) d[i] = 0; return 0; }
int MPI_Cart_shift(MPI_Comm a, int b, int c, int *d, int *e) { (void)a; (void)b; (void)c; *d = *e = MPI_PROC_NULL; return 0; }
int MPI_Type_create_subarray(int a, const int *b, const int *c, const int *d, int e, MPI_Datatype f, MPI_Datatype *g)
{ (void)a; (void)b; (void)c; (void)d; (void)e; *g = f; return 0; }
int MPI_Type_commit(MPI_Datatype *t) { (void)t; return 0; }
int MPI_Type_size(MPI_Datatype t, int *s) { *s = (int)dtype_size(t); return 0; }

#define SHM_FILES 8
static struct { int open, fd; MPI_Offset pos; } g_file[SHM_FILES];

static int file_slot(MPI_File fh) { return fh >= 0 && fh < SHM_FILES && g_file[fh].open ? fh : -1; }

int MPI_File_open(MPI_Comm c, const char *name, int amode, MPI_Info info, MPI_File *fh)
{
    (void)c; (void)info;
    if (amode != MPI_MODE_RDONLY) return 1;
    for (int i = 0; i < SHM_FILES; i++)
        if (!g_file[i].open) {
            const int fd = open(name, O_RDONLY);
            if (fd < 0) return 1;
            g_file[i].open = 1;
            g_file[i].fd = fd;
            g_file[i].pos = 0;
            *fh = i;
            return 0;
        }
    return 1;
}

int MPI_File_get_size(MPI_File fh, MPI_Offset *size)
{
    struct stat st;
    const int i = file_slot(fh);
    if (i < 0 || fstat(g_file[i].fd, &st)) return 1;
    *size = (MPI_Offset)st.st_size;
    return 0;
}

int MPI_File_set_view(MPI_File fh, MPI_Offset disp, MPI_Datatype et, MPI_Datatype ft, const char *rep, MPI_Info info)
{
    (void)info;
    const int i = file_slot(fh);
    if (i < 0 || et != MPI_CHAR || ft != MPI_CHAR || strcmp(rep, "native")) return 1;
    g_file[i].pos = disp;
    return 0;
}

int MPI_File_read(MPI_File fh, void *buf, int n, MPI_Datatype t, MPI_Status *st)
{
    (void)st;
    const int i = file_slot(fh);
    const size_t bytes = (size_t)n * dtype_size(t);
    if (i < 0) return 1;
    const ssize_t got = pread(g_file[i].fd, buf, bytes, (off_t)g_file[i].pos);
    if (got < 0 || (size_t)got != bytes) return 1;
    g_file[i].pos += got;
    return 0;
}

int MPI_File_close(MPI_File *fh)
{
    const int i = file_slot(*fh);
    if (i < 0) return 1;
    close(g_file[i].fd);
    g_file[i].open = 0;
    *fh = -1;
    return 0;
}

/*
 * Run body(rank, arg) on nranks forked processes sharing the mailboxes
 * (slot_bytes: the largest message); the caller only waits, so an abort in
 * a rank cannot take it down.  Returns 0 when every rank returned 0.  Call
 * it from a process that has no GPU context (the children only run host
 * code); results come back through memory the caller mapped MAP_SHARED.
 */
int shm_run(int nranks, size_t slot_bytes, int (*body)(int rank, void *arg), void *arg)
{
    if (nranks < 1 || nranks > 256) return -1;
    const size_t per = sizeof(slot_t) + slot_bytes;
    g_map_bytes = sizeof(shm_head_t) + (size_t)nranks * nranks * SHM_SLOTS * per + (size_t)nranks * SHM_STAGE_BYTES;
    g_base = mmap(NULL, g_map_bytes, PROT_READ | PROT_WRITE, MAP_SHARED | MAP_ANONYMOUS | MAP_NORESERVE, -1, 0);
    if (g_base == MAP_FAILED) return -1;
    g_head = (shm_head_t *)g_base;
    memset(g_head, 0, sizeof *g_head);
    g_head->nranks = nranks;
    g_head->slot_bytes = slot_bytes;
    fflush(stdout);
    fflush(stderr);
    pid_t pid[256];
    int rc = 0;
    for (int r = 0; r < nranks; r++) {
        pid[r] = fork();
        if (pid[r] == 0) {
            g_rank = r;
            g_local_sense = 0;
            int c = body(r, arg);
            fflush(stdout);
            _exit(c ? 1 : 0);
        }
        if (pid[r] < 0) { g_head->abort_code = 1; rc = -1; }
    }
    for (int r = 0; r < nranks; r++) {
        int st = 0;
        if (pid[r] > 0 && (waitpid(pid[r], &st, 0) < 0 || !WIFEXITED(st) || WEXITSTATUS(st) != 0)) rc = -2;
    }
    munmap(g_base, g_map_bytes);
    g_head = NULL;
    g_base = NULL;
    return rc;
}
