/*
 * Single-process MPI for building the reference's own Elemental sources as
 * the CPU oracle (TEST INFRASTRUCTURE ONLY; oracle/refbuild/Makefile).  The
 * reference needs an MPI to compile; the path it is built for runs on one
 * process (a sequential Matrix<F>, or a DistMatrix on a 1 x 1 Grid), where
 * every communicator has size 1 and rank 0.  This header declares the MPI
 * names the reference uses; mpi_single.cpp gives them their size-1 meaning:
 * collectives copy the send buffer to the receive buffer, messages to self
 * are queued, and user reduction operators are never applied (one operand).
 */
#ifndef EREF_SINGLE_MPI_H
#define EREF_SINGLE_MPI_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Group;
typedef int MPI_Errhandler;
typedef int MPI_Request;
typedef struct {
  int MPI_SOURCE;
  int MPI_TAG;
  int MPI_ERROR;
  int count_bytes;
} MPI_Status;
typedef void MPI_User_function(void* invec, void* inoutvec, int* len, MPI_Datatype* datatype);

#define MPI_SUCCESS 0
#define MPI_ERR_OTHER 15
#define MPI_MAX_ERROR_STRING 256

#define MPI_COMM_NULL 0
#define MPI_COMM_WORLD 1
#define MPI_COMM_SELF 2

#define MPI_GROUP_NULL 0
#define MPI_GROUP_EMPTY 1

#define MPI_REQUEST_NULL 0
#define MPI_ERRORS_ARE_FATAL 1
#define MPI_ERRORS_RETURN 2

#define MPI_IDENT 0
#define MPI_CONGRUENT 1
#define MPI_SIMILAR 2
#define MPI_UNEQUAL 3

#define MPI_UNDEFINED (-32766)
#define MPI_ANY_SOURCE (-2)
#define MPI_ANY_TAG (-1)
#define MPI_PROC_NULL (-1)

#define MPI_THREAD_SINGLE 0
#define MPI_THREAD_FUNNELED 1
#define MPI_THREAD_SERIALIZED 2
#define MPI_THREAD_MULTIPLE 3

#define MPI_IN_PLACE ((void*)-1)
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)

/* built-in datatypes (the value encodes nothing; sizes in mpi_single.cpp) */
#define MPI_BYTE 1
#define MPI_CHAR 2
#define MPI_UNSIGNED_CHAR 3
#define MPI_INT 4
#define MPI_UNSIGNED 5
#define MPI_LONG 6
#define MPI_UNSIGNED_LONG 7
#define MPI_LONG_LONG_INT 8
#define MPI_UNSIGNED_LONG_LONG 9
#define MPI_FLOAT 10
#define MPI_DOUBLE 11
#define MPI_COMPLEX 12
#define MPI_DOUBLE_COMPLEX 13
#define MPI_FLOAT_INT 14
#define MPI_DOUBLE_INT 15
#define MPI_2INT 16
#define MPI_LONG_LONG MPI_LONG_LONG_INT

/* built-in operators; created operators are numbered from 100 */
#define MPI_OP_NULL 0
#define MPI_MAX 1
#define MPI_MIN 2
#define MPI_SUM 3
#define MPI_PROD 4
#define MPI_LAND 5
#define MPI_BAND 6
#define MPI_LOR 7
#define MPI_BOR 8
#define MPI_LXOR 9
#define MPI_BXOR 10
#define MPI_MAXLOC 11
#define MPI_MINLOC 12

int MPI_Init(int* argc, char*** argv);
int MPI_Init_thread(int* argc, char*** argv, int required, int* provided);
int MPI_Initialized(int* flag);
int MPI_Finalized(int* flag);
int MPI_Finalize(void);
int MPI_Query_thread(int* provided);
double MPI_Wtime(void);
int MPI_Error_string(int errorcode, char* string, int* resultlen);
int MPI_Errhandler_set(MPI_Comm comm, MPI_Errhandler handler);
int MPI_Comm_set_errhandler(MPI_Comm comm, MPI_Errhandler handler);

int MPI_Comm_size(MPI_Comm comm, int* size);
int MPI_Comm_rank(MPI_Comm comm, int* rank);
int MPI_Comm_dup(MPI_Comm comm, MPI_Comm* newcomm);
int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm* newcomm);
int MPI_Comm_create(MPI_Comm comm, MPI_Group group, MPI_Comm* newcomm);
int MPI_Comm_free(MPI_Comm* comm);
int MPI_Comm_compare(MPI_Comm a, MPI_Comm b, int* result);
int MPI_Comm_group(MPI_Comm comm, MPI_Group* group);
int MPI_Cart_create(MPI_Comm comm, int ndims, const int* dims, const int* periods, int reorder, MPI_Comm* cart);
int MPI_Cart_sub(MPI_Comm comm, const int* remain_dims, MPI_Comm* newcomm);

int MPI_Group_size(MPI_Group group, int* size);
int MPI_Group_rank(MPI_Group group, int* rank);
int MPI_Group_incl(MPI_Group group, int n, const int* ranks, MPI_Group* newgroup);
int MPI_Group_difference(MPI_Group a, MPI_Group b, MPI_Group* newgroup);
int MPI_Group_translate_ranks(MPI_Group a, int n, const int* ranks_a, MPI_Group b, int* ranks_b);
int MPI_Group_free(MPI_Group* group);

int MPI_Op_create(MPI_User_function* fn, int commute, MPI_Op* op);
int MPI_Op_free(MPI_Op* op);

int MPI_Send(const void* buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm);
int MPI_Recv(void* buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm comm, MPI_Status* status);
int MPI_Isend(const void* buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm, MPI_Request* req);
int MPI_Issend(const void* buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm, MPI_Request* req);
int MPI_Irecv(void* buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm comm, MPI_Request* req);
int MPI_Sendrecv(const void* sbuf, int scount, MPI_Datatype stype, int dest, int stag, void* rbuf, int rcount,
                 MPI_Datatype rtype, int source, int rtag, MPI_Comm comm, MPI_Status* status);
int MPI_Sendrecv_replace(void* buf, int count, MPI_Datatype type, int dest, int stag, int source, int rtag,
                         MPI_Comm comm, MPI_Status* status);
int MPI_Iprobe(int source, int tag, MPI_Comm comm, int* flag, MPI_Status* status);
int MPI_Get_count(const MPI_Status* status, MPI_Datatype type, int* count);
int MPI_Test(MPI_Request* req, int* flag, MPI_Status* status);
int MPI_Wait(MPI_Request* req, MPI_Status* status);
int MPI_Waitall(int count, MPI_Request* reqs, MPI_Status* statuses);

int MPI_Barrier(MPI_Comm comm);
int MPI_Bcast(void* buf, int count, MPI_Datatype type, int root, MPI_Comm comm);
int MPI_Ibcast(void* buf, int count, MPI_Datatype type, int root, MPI_Comm comm, MPI_Request* req);
int MPI_Gather(const void* sbuf, int scount, MPI_Datatype stype, void* rbuf, int rcount, MPI_Datatype rtype, int root,
               MPI_Comm comm);
int MPI_Igather(const void* sbuf, int scount, MPI_Datatype stype, void* rbuf, int rcount, MPI_Datatype rtype,
                int root, MPI_Comm comm, MPI_Request* req);
int MPI_Gatherv(const void* sbuf, int scount, MPI_Datatype stype, void* rbuf, const int* rcounts, const int* displs,
                MPI_Datatype rtype, int root, MPI_Comm comm);
int MPI_Allgather(const void* sbuf, int scount, MPI_Datatype stype, void* rbuf, int rcount, MPI_Datatype rtype,
                  MPI_Comm comm);
int MPI_Allgatherv(const void* sbuf, int scount, MPI_Datatype stype, void* rbuf, const int* rcounts,
                   const int* displs, MPI_Datatype rtype, MPI_Comm comm);
int MPI_Scatter(const void* sbuf, int scount, MPI_Datatype stype, void* rbuf, int rcount, MPI_Datatype rtype,
                int root, MPI_Comm comm);
int MPI_Alltoall(const void* sbuf, int scount, MPI_Datatype stype, void* rbuf, int rcount, MPI_Datatype rtype,
                 MPI_Comm comm);
int MPI_Alltoallv(const void* sbuf, const int* scounts, const int* sdispls, MPI_Datatype stype, void* rbuf,
                  const int* rcounts, const int* rdispls, MPI_Datatype rtype, MPI_Comm comm);
int MPI_Reduce(const void* sbuf, void* rbuf, int count, MPI_Datatype type, MPI_Op op, int root, MPI_Comm comm);
int MPI_Allreduce(const void* sbuf, void* rbuf, int count, MPI_Datatype type, MPI_Op op, MPI_Comm comm);
int MPI_Reduce_scatter(const void* sbuf, void* rbuf, const int* rcounts, MPI_Datatype type, MPI_Op op,
                       MPI_Comm comm);
int MPI_Reduce_scatter_block(const void* sbuf, void* rbuf, int rcount, MPI_Datatype type, MPI_Op op,
                             MPI_Comm comm);

#ifdef __cplusplus
}
#endif

#endif /* EREF_SINGLE_MPI_H */
