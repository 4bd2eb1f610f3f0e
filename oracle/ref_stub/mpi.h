/*
 * Serial, single-rank stand-in for <mpi.h>.
 *
 * Test infrastructure only: it lets the unmodified reference library
 * (dmhm, compiled by oracle/Makefile) link without an MPI installation so it
 * can serve as the CPU correctness oracle and the timed CPU baseline.  Every
 * communicator has exactly one rank; collectives copy the send buffer into
 * the receive buffer; point-to-point calls are not supported (the serial
 * HMat2d/HMat3d paths and single-rank DistHMat never reach them with a peer).
 * The symbols are the ones the reference uses in src/core/mpi.cpp.
 */
#ifndef ORACLE_SERIAL_MPI_H
#define ORACLE_SERIAL_MPI_H 1

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Datatype;   /* value = element size in bytes */
typedef int MPI_Errhandler;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR, count; } MPI_Status;

#define MPI_SUCCESS 0
#define MPI_ANY_SOURCE (-1)
#define MPI_ANY_TAG (-1)
#define MPI_UNDEFINED (-32766)
#define MPI_COMM_WORLD ((MPI_Comm)1)
#define MPI_COMM_SELF ((MPI_Comm)2)
#define MPI_ERRORS_RETURN ((MPI_Errhandler)1)
#define MPI_ERRORS_ARE_FATAL ((MPI_Errhandler)2)
#define MPI_REQUEST_NULL ((MPI_Request)0)
#define MPI_IN_PLACE ((void*)1)
#define MPI_MAX_ERROR_STRING 256

#define MPI_MAX 1
#define MPI_MIN 2
#define MPI_MAXLOC 3
#define MPI_MINLOC 4
#define MPI_PROD 5
#define MPI_SUM 6
#define MPI_LAND 7
#define MPI_LOR 8
#define MPI_LXOR 9
#define MPI_BAND 10
#define MPI_BOR 11
#define MPI_BXOR 12

#define MPI_BYTE ((MPI_Datatype)1)
#define MPI_UNSIGNED_CHAR ((MPI_Datatype)1)
#define MPI_CHAR ((MPI_Datatype)1)
#define MPI_INT ((MPI_Datatype)4)
#define MPI_UNSIGNED ((MPI_Datatype)4)
#define MPI_FLOAT ((MPI_Datatype)4)
#define MPI_DOUBLE ((MPI_Datatype)8)
#define MPI_LONG_LONG_INT ((MPI_Datatype)8)
#define MPI_COMPLEX ((MPI_Datatype)8)
#define MPI_DOUBLE_COMPLEX ((MPI_Datatype)16)
#define MPI_2INT ((MPI_Datatype)8)
#define MPI_FLOAT_INT ((MPI_Datatype)8)
#define MPI_DOUBLE_INT ((MPI_Datatype)12)

int MPI_Init(int* argc, char*** argv);
int MPI_Finalize(void);
int MPI_Initialized(int* flag);
int MPI_Finalized(int* flag);
double MPI_Wtime(void);
int MPI_Abort(MPI_Comm comm, int code);
int MPI_Error_string(int code, char* str, int* len);
int MPI_Comm_rank(MPI_Comm comm, int* rank);
int MPI_Comm_size(MPI_Comm comm, int* size);
int MPI_Comm_dup(MPI_Comm comm, MPI_Comm* out);
int MPI_Comm_free(MPI_Comm* comm);
int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm* out);
int MPI_Send(void* buf, int count, MPI_Datatype t, int to, int tag, MPI_Comm c);
int MPI_Recv(void* buf, int count, MPI_Datatype t, int from, int tag,
             MPI_Comm c, MPI_Status* st);
int MPI_Isend(void* buf, int count, MPI_Datatype t, int to, int tag,
              MPI_Comm c, MPI_Request* req);
int MPI_Irecv(void* buf, int count, MPI_Datatype t, int from, int tag,
              MPI_Comm c, MPI_Request* req);
int MPI_Wait(MPI_Request* req, MPI_Status* st);
int MPI_Waitall(int n, MPI_Request* reqs, MPI_Status* sts);
int MPI_Barrier(MPI_Comm c);
int MPI_Bcast(void* buf, int count, MPI_Datatype t, int root, MPI_Comm c);
int MPI_Reduce(void* sbuf, void* rbuf, int count, MPI_Datatype t, MPI_Op op,
               int root, MPI_Comm c);
int MPI_Allreduce(void* sbuf, void* rbuf, int count, MPI_Datatype t,
                  MPI_Op op, MPI_Comm c);
int MPI_Allgather(void* sbuf, int scount, MPI_Datatype st, void* rbuf,
                  int rcount, MPI_Datatype rt, MPI_Comm c);
int MPI_Alltoall(void* sbuf, int scount, MPI_Datatype st, void* rbuf,
                 int rcount, MPI_Datatype rt, MPI_Comm c);
int MPI_Sendrecv(void* sbuf, int scount, MPI_Datatype st, int to, int stag,
                 void* rbuf, int rcount, MPI_Datatype rt, int from, int rtag,
                 MPI_Comm c, MPI_Status* status);

#ifdef __cplusplus
}
#endif
#endif
