/*
 * Single-rank implementation of the serial <mpi.h> stand-in (test
 * infrastructure for the reference oracle; see mpi.h in this folder).
 */
#include "mpi.h"
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

static int g_init = 0, g_fin = 0;

int MPI_Init(int* argc, char*** argv) { (void)argc; (void)argv; g_init = 1; return 0; }
int MPI_Finalize(void) { g_fin = 1; return 0; }
int MPI_Initialized(int* flag) { *flag = g_init; return 0; }
int MPI_Finalized(int* flag) { *flag = g_fin; return 0; }
double MPI_Wtime(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}
int MPI_Abort(MPI_Comm comm, int code) { (void)comm; exit(code); }
int MPI_Error_string(int code, char* str, int* len)
{
    *len = snprintf(str, MPI_MAX_ERROR_STRING, "serial MPI stub error %d", code);
    return 0;
}
int MPI_Comm_rank(MPI_Comm comm, int* rank) { (void)comm; *rank = 0; return 0; }
int MPI_Comm_size(MPI_Comm comm, int* size) { (void)comm; *size = 1; return 0; }
int MPI_Comm_dup(MPI_Comm comm, MPI_Comm* out) { *out = comm; return 0; }
int MPI_Comm_free(MPI_Comm* comm) { (void)comm; return 0; }
int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm* out)
{ (void)color; (void)key; *out = comm; return 0; }

static void unsupported(const char* what)
{
    fprintf(stderr, "serial MPI stub: %s with a peer is not supported\n", what);
    abort();
}
int MPI_Send(void* b, int n, MPI_Datatype t, int to, int tag, MPI_Comm c)
{ (void)b; (void)n; (void)t; (void)to; (void)tag; (void)c; unsupported("MPI_Send"); return 1; }
int MPI_Recv(void* b, int n, MPI_Datatype t, int f, int tag, MPI_Comm c, MPI_Status* s)
{ (void)b; (void)n; (void)t; (void)f; (void)tag; (void)c; (void)s; unsupported("MPI_Recv"); return 1; }
int MPI_Isend(void* b, int n, MPI_Datatype t, int to, int tag, MPI_Comm c, MPI_Request* r)
{ (void)b; (void)n; (void)t; (void)to; (void)tag; (void)c; (void)r; unsupported("MPI_Isend"); return 1; }
int MPI_Irecv(void* b, int n, MPI_Datatype t, int f, int tag, MPI_Comm c, MPI_Request* r)
{ (void)b; (void)n; (void)t; (void)f; (void)tag; (void)c; (void)r; unsupported("MPI_Irecv"); return 1; }
int MPI_Wait(MPI_Request* r, MPI_Status* s) { (void)r; (void)s; return 0; }
int MPI_Waitall(int n, MPI_Request* r, MPI_Status* s) { (void)n; (void)r; (void)s; return 0; }
int MPI_Barrier(MPI_Comm c) { (void)c; return 0; }
int MPI_Bcast(void* b, int n, MPI_Datatype t, int root, MPI_Comm c)
{ (void)b; (void)n; (void)t; (void)root; (void)c; return 0; }

static void copy_in(void* s, void* r, size_t bytes)
{
    if (s != MPI_IN_PLACE && s != r && r != 0 && bytes) memmove(r, s, bytes);
}
int MPI_Reduce(void* s, void* r, int n, MPI_Datatype t, MPI_Op op, int root, MPI_Comm c)
{ (void)op; (void)root; (void)c; copy_in(s, r, (size_t)n * (size_t)t); return 0; }
int MPI_Allreduce(void* s, void* r, int n, MPI_Datatype t, MPI_Op op, MPI_Comm c)
{ (void)op; (void)c; copy_in(s, r, (size_t)n * (size_t)t); return 0; }
int MPI_Allgather(void* s, int sn, MPI_Datatype st, void* r, int rn, MPI_Datatype rt, MPI_Comm c)
{ (void)rn; (void)rt; (void)c; copy_in(s, r, (size_t)sn * (size_t)st); return 0; }
int MPI_Alltoall(void* s, int sn, MPI_Datatype st, void* r, int rn, MPI_Datatype rt, MPI_Comm c)
{ (void)rn; (void)rt; (void)c; copy_in(s, r, (size_t)sn * (size_t)st); return 0; }
int MPI_Sendrecv(void* s, int sn, MPI_Datatype st, int to, int stag, void* r, int rn,
                 MPI_Datatype rt, int from, int rtag, MPI_Comm c, MPI_Status* status)
{
    (void)rn; (void)rt; (void)stag; (void)rtag; (void)c; (void)status;
    if (to != 0 || from != 0) unsupported("MPI_Sendrecv");
    copy_in(s, r, (size_t)sn * (size_t)st);
    return 0;
}
