/*
 * One-process MPI for the translated reference program -- TEST INFRASTRUCTURE ONLY.
 *
 * The reference (t3dsdsc.f) is an MPI program; at a 1x1 process grid (nprx = nprz = 1) every
 * neighbour rank is MPI_PROC_NULL (the main program's set-up, t3dsdsc.f:46-55), so halo
 * exchanges move nothing, reductions and gathers over one rank are copies, and barriers and
 * derived types have no effect.  Each routine receives the number of Fortran arguments and
 * then their addresses (arguments by reference), as f77c.py emits the calls.  The constants
 * match f77c.py's mpif.h table.
 */
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

enum { COMM_WORLD = 91, PROC_NULL = -2, T_DOUBLE = 11, T_INTEGER = 7, T_REAL = 10, T_LOGICAL = 8,
       T_CHARACTER = 9 };

static long type_size(int t) {
    switch (t) {
        case T_DOUBLE: return 8;
        case T_INTEGER: case T_REAL: case T_LOGICAL: return 4;
        case T_CHARACTER: return 1;
        default:
            fprintf(stderr, "mpi stub: derived datatype %d in a data transfer\n", t);
            abort();
    }
}

void ref_unreachable(const char* what) {
    fprintf(stderr, "translated reference: reached a statement that was not translated: %s\n", what);
    abort();
}

void ref_stop(const char* where) {
    fprintf(stderr, "translated reference: STOP in %s\n", where);
    abort();
}

#define ARGS(n, a)                                                      \
    void* a[16];                                                        \
    do {                                                                \
        va_list ap;                                                     \
        va_start(ap, n);                                                \
        for (int q = 0; q < n && q < 16; ++q) a[q] = va_arg(ap, void*); \
        va_end(ap);                                                     \
    } while (0)
#define IERR(a, q) (*(int*)(a)[q] = 0)

void f_mpi_init(int n, ...) { ARGS(n, a); IERR(a, 0); }
void f_mpi_finalize(int n, ...) { ARGS(n, a); IERR(a, 0); }
void f_mpi_barrier(int n, ...) { ARGS(n, a); IERR(a, 1); }
void f_mpi_comm_size(int n, ...) { ARGS(n, a); *(int*)a[1] = 1; IERR(a, 2); }
void f_mpi_comm_rank(int n, ...) { ARGS(n, a); *(int*)a[1] = 0; IERR(a, 2); }
void f_mpi_abort(int n, ...) { (void)n; fprintf(stderr, "mpi stub: MPI_ABORT\n"); abort(); }

/* allreduce(send, recv, count, type, op, comm, ierr) over one rank: recv = send */
void f_mpi_allreduce(int n, ...) {
    ARGS(n, a);
    long bytes = (long)*(int*)a[2] * type_size(*(int*)a[3]);
    if (a[0] != a[1]) memmove(a[1], a[0], (size_t)bytes);
    IERR(a, 6);
}
/* reduce(send, recv, count, type, op, root, comm, ierr) */
void f_mpi_reduce(int n, ...) {
    ARGS(n, a);
    long bytes = (long)*(int*)a[2] * type_size(*(int*)a[3]);
    if (a[0] != a[1]) memmove(a[1], a[0], (size_t)bytes);
    IERR(a, 7);
}
/* gather(send, scount, stype, recv, rcount, rtype, root, comm, ierr) */
void f_mpi_gather(int n, ...) {
    ARGS(n, a);
    long bytes = (long)*(int*)a[1] * type_size(*(int*)a[2]);
    if (a[0] != a[3]) memmove(a[3], a[0], (size_t)bytes);
    IERR(a, 8);
}
/* send(buf, count, type, dest, tag, comm, ierr) / recv(buf, count, type, source, tag, comm,
 * status, ierr): only MPI_PROC_NULL partners exist in a one-process run */
void f_mpi_send(int n, ...) {
    ARGS(n, a);
    if (*(int*)a[3] != PROC_NULL) { fprintf(stderr, "mpi stub: send to rank %d\n", *(int*)a[3]); abort(); }
    IERR(a, 6);
}
void f_mpi_recv(int n, ...) {
    ARGS(n, a);
    if (*(int*)a[3] != PROC_NULL) { fprintf(stderr, "mpi stub: recv from rank %d\n", *(int*)a[3]); abort(); }
    IERR(a, 7);
}
/* sendrecv(sbuf, scount, stype, dest, stag, rbuf, rcount, rtype, source, rtag, comm, status, ierr) */
void f_mpi_sendrecv(int n, ...) {
    ARGS(n, a);
    if (*(int*)a[3] != PROC_NULL || *(int*)a[8] != PROC_NULL) {
        fprintf(stderr, "mpi stub: sendrecv with ranks %d / %d\n", *(int*)a[3], *(int*)a[8]);
        abort();
    }
    IERR(a, 12);
}
static int next_type = 1000;
/* type_contiguous(count, oldtype, newtype, ierr); type_vector(count, blocklen, stride, oldtype,
 * newtype, ierr) */
void f_mpi_type_contiguous(int n, ...) { ARGS(n, a); *(int*)a[2] = next_type++; IERR(a, 3); }
void f_mpi_type_vector(int n, ...) { ARGS(n, a); *(int*)a[4] = next_type++; IERR(a, 5); }
void f_mpi_type_commit(int n, ...) { ARGS(n, a); IERR(a, 1); }
void f_mpi_type_free(int n, ...) { ARGS(n, a); IERR(a, 1); }
