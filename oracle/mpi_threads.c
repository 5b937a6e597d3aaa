/*
 * MPI for ranks that are threads of one process -- TEST INFRASTRUCTURE ONLY.
 *
 * The translated reference built with -DREF_TLS=__thread keeps every COMMON block and static
 * local array per thread, so each thread can run as one rank of the reference's nprx x nprz
 * decomposition (t3dsdsc.f:33-81).  This file gives those ranks the MPI calls the reference
 * makes: point-to-point messages (sendrecv, send, recv; buffered sends, so that the reference's
 * exchange order cannot deadlock), the contiguous and vector datatypes of its halo messages
 * (message1..message5, t3dsdsc.f:6170-6485), barrier, and allreduce / reduce / gather over all
 * ranks, reduced in rank order so that results do not depend on thread timing.  The same
 * argument convention as mpi_stub.c: the count of Fortran arguments, then their addresses.
 */
#include <pthread.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

enum { PROC_NULL = -2, T_DOUBLE = 11, T_INTEGER = 7, T_REAL = 10, T_LOGICAL = 8, T_CHARACTER = 9,
       OP_MIN = 101, OP_MAX = 102, OP_SUM = 103 };

static __thread int my_rank = 0;
static int n_ranks = 1;
static pthread_barrier_t bar;

void mpt_set_rank(int r) { my_rank = r; }
void mpt_init(int n) { n_ranks = n; pthread_barrier_init(&bar, NULL, (unsigned)n); }
void mpt_fini(void) { pthread_barrier_destroy(&bar); }
void mpt_barrier(void) { pthread_barrier_wait(&bar); }

void ref_unreachable(const char* what) {
    fprintf(stderr, "translated reference: reached a statement that was not translated: %s\n", what);
    abort();
}
void ref_stop(const char* where) {
    fprintf(stderr, "translated reference: STOP in %s\n", where);
    abort();
}

/* ---- datatypes: contiguous(count, old) and vector(count, blocklen, stride, old) of doubles ---- */
typedef struct { int used, kind, count, blocklen, stride, old; } dtype;
static dtype types[4096];
static pthread_mutex_t types_mu = PTHREAD_MUTEX_INITIALIZER;

static long base_size(int t) {
    switch (t) {
        case T_DOUBLE: return 8;
        case T_INTEGER: case T_REAL: case T_LOGICAL: return 4;
        case T_CHARACTER: return 1;
        default: return 0;
    }
}
/* bytes of `count` items of type t packed */
static long packed_bytes(int t, int count) {
    long b = base_size(t);
    if (b) return b * count;
    if (t < 1000 || t >= 1000 + 4096 || !types[t - 1000].used) { fprintf(stderr, "mpi: bad type %d\n", t); abort(); }
    const dtype* d = &types[t - 1000];
    long one = d->kind == 0 ? packed_bytes(d->old, d->count) : (long)d->count * packed_bytes(d->old, d->blocklen);
    return one * count;
}
static long extent_elems(const dtype* d) {   /* extent of one item, in elements of `old` */
    return d->kind == 0 ? d->count : (long)(d->count - 1) * d->stride + d->blocklen;
}
static void pack(char* dst, const char* src, int t, int count) {
    long b = base_size(t);
    if (b) { memcpy(dst, src, (size_t)(b * count)); return; }
    const dtype* d = &types[t - 1000];
    long ob = packed_bytes(d->old, 1), ext = extent_elems(d) * ob;
    for (int c = 0; c < count; ++c, src += ext) {
        if (d->kind == 0) { pack(dst, src, d->old, d->count); dst += ob * d->count; }
        else for (int q = 0; q < d->count; ++q) { pack(dst, src + (long)q * d->stride * ob, d->old, d->blocklen); dst += ob * d->blocklen; }
    }
}
static void unpack(char* dst, const char* src, int t, int count) {
    long b = base_size(t);
    if (b) { memcpy(dst, src, (size_t)(b * count)); return; }
    const dtype* d = &types[t - 1000];
    long ob = packed_bytes(d->old, 1), ext = extent_elems(d) * ob;
    for (int c = 0; c < count; ++c, dst += ext) {
        if (d->kind == 0) { unpack(dst, src, d->old, d->count); src += ob * d->count; }
        else for (int q = 0; q < d->count; ++q) { unpack(dst + (long)q * d->stride * ob, src, d->old, d->blocklen); src += ob * d->blocklen; }
    }
}
static int new_type(dtype d) {
    pthread_mutex_lock(&types_mu);
    int h = -1;
    for (int q = 0; q < 4096; ++q) if (!types[q].used) { types[q] = d; types[q].used = 1; h = 1000 + q; break; }
    pthread_mutex_unlock(&types_mu);
    if (h < 0) { fprintf(stderr, "mpi: out of datatypes\n"); abort(); }
    return h;
}

/* ---- buffered point-to-point messages: a list per destination rank ---- */
typedef struct msg { int src, tag; long bytes; char* data; struct msg* next; } msg;
typedef struct { pthread_mutex_t mu; pthread_cond_t cv; msg* head; } mailbox;
static mailbox boxes[1024];
static pthread_once_t boxes_once = PTHREAD_ONCE_INIT;
static void boxes_init(void) {
    for (int q = 0; q < 1024; ++q) { pthread_mutex_init(&boxes[q].mu, NULL); pthread_cond_init(&boxes[q].cv, NULL); boxes[q].head = NULL; }
}
static void post(int dest, int tag, const void* buf, int count, int t) {
    pthread_once(&boxes_once, boxes_init);
    msg* m = (msg*)malloc(sizeof(msg));
    m->src = my_rank; m->tag = tag; m->bytes = packed_bytes(t, count);
    m->data = (char*)malloc((size_t)m->bytes + 1);
    pack(m->data, (const char*)buf, t, count);
    m->next = NULL;
    mailbox* b = &boxes[dest];
    pthread_mutex_lock(&b->mu);
    msg** p = &b->head;
    while (*p) p = &(*p)->next;   /* FIFO per (source, tag): MPI's non-overtaking order */
    *p = m;
    pthread_cond_broadcast(&b->cv);
    pthread_mutex_unlock(&b->mu);
}
static void take(int src, int tag, void* buf, int count, int t) {
    pthread_once(&boxes_once, boxes_init);
    mailbox* b = &boxes[my_rank];
    pthread_mutex_lock(&b->mu);
    for (;;) {
        for (msg** p = &b->head; *p; p = &(*p)->next)
            if ((*p)->src == src && (*p)->tag == tag) {
                msg* m = *p;
                *p = m->next;
                pthread_mutex_unlock(&b->mu);
                if (m->bytes != packed_bytes(t, count)) { fprintf(stderr, "mpi: message size mismatch\n"); abort(); }
                unpack((char*)buf, m->data, t, count);
                free(m->data);
                free(m);
                return;
            }
        pthread_cond_wait(&b->cv, &b->mu);
    }
}

/* ---- collectives: every rank writes its contribution, reduce in rank order ---- */
static void* slots[1024];
static void reduce_all(const void* send, void* recv, int count, int t, int op, int root /* -1: all */) {
    slots[my_rank] = (void*)send;
    pthread_barrier_wait(&bar);
    if (root < 0 || my_rank == root) {
        long n = count;
        if (t == T_DOUBLE) {
            double* acc = (double*)malloc(sizeof(double) * (size_t)n);
            memcpy(acc, slots[0], sizeof(double) * (size_t)n);
            for (int r = 1; r < n_ranks; ++r) {
                const double* v = (const double*)slots[r];
                for (long q = 0; q < n; ++q)
                    acc[q] = op == OP_MIN ? (v[q] < acc[q] ? v[q] : acc[q]) : op == OP_MAX ? (v[q] > acc[q] ? v[q] : acc[q]) : acc[q] + v[q];
            }
            pthread_barrier_wait(&bar);   /* every rank has read the slots before any writes recv */
            memcpy(recv, acc, sizeof(double) * (size_t)n);
            free(acc);
        } else if (t == T_INTEGER || t == T_LOGICAL) {
            int* acc = (int*)malloc(sizeof(int) * (size_t)n);
            memcpy(acc, slots[0], sizeof(int) * (size_t)n);
            for (int r = 1; r < n_ranks; ++r) {
                const int* v = (const int*)slots[r];
                for (long q = 0; q < n; ++q)
                    acc[q] = op == OP_MIN ? (v[q] < acc[q] ? v[q] : acc[q]) : op == OP_MAX ? (v[q] > acc[q] ? v[q] : acc[q]) : acc[q] + v[q];
            }
            pthread_barrier_wait(&bar);
            memcpy(recv, acc, sizeof(int) * (size_t)n);
            free(acc);
        } else { fprintf(stderr, "mpi: reduction of type %d\n", t); abort(); }
    } else {
        pthread_barrier_wait(&bar);
    }
    pthread_barrier_wait(&bar);
}

#define ARGS(n, a)                                                      \
    void* a[16];                                                        \
    do {                                                                \
        va_list ap;                                                     \
        va_start(ap, n);                                                \
        for (int q = 0; q < n && q < 16; ++q) a[q] = va_arg(ap, void*); \
        va_end(ap);                                                     \
    } while (0)
#define I(a, q) (*(int*)(a)[q])
#define IERR(a, q) (*(int*)(a)[q] = 0)

void f_mpi_init(int n, ...) { ARGS(n, a); IERR(a, 0); }
void f_mpi_finalize(int n, ...) { ARGS(n, a); IERR(a, 0); }
void f_mpi_barrier(int n, ...) { ARGS(n, a); pthread_barrier_wait(&bar); IERR(a, 1); }
void f_mpi_comm_size(int n, ...) { ARGS(n, a); I(a, 1) = n_ranks; IERR(a, 2); }
void f_mpi_comm_rank(int n, ...) { ARGS(n, a); I(a, 1) = my_rank; IERR(a, 2); }
void f_mpi_abort(int n, ...) { (void)n; fprintf(stderr, "mpi: MPI_ABORT\n"); abort(); }
/* allreduce(send, recv, count, type, op, comm, ierr) */
void f_mpi_allreduce(int n, ...) { ARGS(n, a); reduce_all(a[0], a[1], I(a, 2), I(a, 3), I(a, 4), -1); IERR(a, 6); }
/* reduce(send, recv, count, type, op, root, comm, ierr) */
void f_mpi_reduce(int n, ...) { ARGS(n, a); reduce_all(a[0], a[1], I(a, 2), I(a, 3), I(a, 4), I(a, 5)); IERR(a, 7); }
/* gather(send, scount, stype, recv, rcount, rtype, root, comm, ierr): rank r's items at r * rcount */
void f_mpi_gather(int n, ...) {
    ARGS(n, a);
    slots[my_rank] = a[0];
    pthread_barrier_wait(&bar);
    if (my_rank == I(a, 6)) {
        long rb = packed_bytes(I(a, 5), I(a, 4));
        for (int r = 0; r < n_ranks; ++r) {
            char* tmp = (char*)malloc((size_t)rb);
            pack(tmp, (const char*)slots[r], I(a, 2), I(a, 1));
            unpack((char*)a[3] + (long)r * rb, tmp, I(a, 5), I(a, 4));
            free(tmp);
        }
    }
    pthread_barrier_wait(&bar);
    IERR(a, 8);
}
/* send(buf, count, type, dest, tag, comm, ierr) */
void f_mpi_send(int n, ...) { ARGS(n, a); if (I(a, 3) != PROC_NULL) post(I(a, 3), I(a, 4), a[0], I(a, 1), I(a, 2)); IERR(a, 6); }
/* recv(buf, count, type, source, tag, comm, status, ierr) */
void f_mpi_recv(int n, ...) { ARGS(n, a); if (I(a, 3) != PROC_NULL) take(I(a, 3), I(a, 4), a[0], I(a, 1), I(a, 2)); IERR(a, 7); }
/* sendrecv(sbuf, scount, stype, dest, stag, rbuf, rcount, rtype, source, rtag, comm, status, ierr) */
void f_mpi_sendrecv(int n, ...) {
    ARGS(n, a);
    if (I(a, 3) != PROC_NULL) post(I(a, 3), I(a, 4), a[0], I(a, 1), I(a, 2));
    if (I(a, 8) != PROC_NULL) take(I(a, 8), I(a, 9), a[5], I(a, 6), I(a, 7));
    IERR(a, 12);
}
/* type_contiguous(count, old, new, ierr); type_vector(count, blocklen, stride, old, new, ierr) */
void f_mpi_type_contiguous(int n, ...) {
    ARGS(n, a);
    dtype d = {1, 0, I(a, 0), 0, 0, I(a, 1)};
    I(a, 2) = new_type(d);
    IERR(a, 3);
}
void f_mpi_type_vector(int n, ...) {
    ARGS(n, a);
    dtype d = {1, 1, I(a, 0), I(a, 1), I(a, 2), I(a, 3)};
    I(a, 4) = new_type(d);
    IERR(a, 5);
}
void f_mpi_type_commit(int n, ...) { ARGS(n, a); IERR(a, 1); }
void f_mpi_type_free(int n, ...) {
    ARGS(n, a);
    int h = I(a, 0);
    if (h >= 1000 && h < 1000 + 4096) { pthread_mutex_lock(&types_mu); types[h - 1000].used = 0; pthread_mutex_unlock(&types_mu); }
    IERR(a, 1);
}
