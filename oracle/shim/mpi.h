/*
 * Size-1 MPI shim for building the reference's dense HOOI as a CPU oracle.
 *
 * Test infrastructure only: this header lets the reference's unmodified
 * sources (communicator.tpp, distribution.cpp, tensor.tpp, ...) compile and
 * run as a single-process world, which is the "mpirun -np 1" case of the
 * reference.  Every collective degenerates to the identity (a copy from the
 * send buffer to the receive buffer where they differ); point-to-point calls
 * are never reached at size 1 (the ring loops in Function::gram /
 * Function::ttt_except skip them when the fibre has one process) and abort if
 * they are.
 */
#ifndef DT_ORACLE_MPI_SHIM_H
#define DT_ORACLE_MPI_SHIM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Op;
typedef int MPI_Request;
/* A datatype is encoded as its element size in bytes (plus a tag bit so that
 * equal-size types stay distinct for debugging). */
typedef int MPI_Datatype;
typedef struct {
    int MPI_SOURCE, MPI_TAG, MPI_ERROR;
} MPI_Status;

#define MPI_COMM_WORLD ((MPI_Comm)0)
#define MPI_COMM_NULL ((MPI_Comm)-1)
#define MPI_SUCCESS 0
#define MPI_SUM ((MPI_Op)1)
#define MPI_MAX ((MPI_Op)2)
#define MPI_MIN ((MPI_Op)3)
#define MPI_PROD ((MPI_Op)4)
#define MPI_THREAD_SINGLE 0
#define MPI_THREAD_FUNNELED 1
#define MPI_THREAD_SERIALIZED 2
#define MPI_THREAD_MULTIPLE 3
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)
#define MPI_IN_PLACE ((void *)1)
#define MPI_REQUEST_NULL ((MPI_Request)0)

#define DT_MPI_TYPE(sz, tag) ((MPI_Datatype)(((tag) << 8) | (sz)))
#define MPI_CHAR DT_MPI_TYPE(1, 1)
#define MPI_UNSIGNED_CHAR DT_MPI_TYPE(1, 2)
#define MPI_UNSIGNED_SHORT DT_MPI_TYPE(2, 3)
#define MPI_INT DT_MPI_TYPE(4, 4)
#define MPI_UNSIGNED DT_MPI_TYPE(4, 5)
#define MPI_FLOAT DT_MPI_TYPE(4, 6)
#define MPI_LONG DT_MPI_TYPE(8, 7)
#define MPI_UNSIGNED_LONG DT_MPI_TYPE(8, 8)
#define MPI_LONG_LONG_INT DT_MPI_TYPE(8, 9)
#define MPI_LONG_LONG DT_MPI_TYPE(8, 9)
#define MPI_UNSIGNED_LONG_LONG DT_MPI_TYPE(8, 10)
#define MPI_DOUBLE DT_MPI_TYPE(8, 11)
#define MPI_C_COMPLEX DT_MPI_TYPE(8, 12)
#define MPI_C_DOUBLE_COMPLEX DT_MPI_TYPE(16, 13)

int MPI_Init(int *argc, char ***argv);
int MPI_Init_thread(int *argc, char ***argv, int required, int *provided);
int MPI_Finalize(void);
int MPI_Abort(MPI_Comm comm, int code);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm *newcomm);
double MPI_Wtime(void);
int MPI_Barrier(MPI_Comm comm);
int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root, MPI_Comm comm);
int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype type,
                  MPI_Op op, MPI_Comm comm);
int MPI_Iallreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype type,
                   MPI_Op op, MPI_Comm comm, MPI_Request *req);
int MPI_Reduce_scatter(const void *sendbuf, void *recvbuf, const int *recvcounts,
                       MPI_Datatype type, MPI_Op op, MPI_Comm comm);
int MPI_Allgather(const void *sendbuf, int sendcount, MPI_Datatype sendtype,
                  void *recvbuf, int recvcount, MPI_Datatype recvtype, MPI_Comm comm);
int MPI_Allgatherv(const void *sendbuf, int sendcount, MPI_Datatype sendtype,
                   void *recvbuf, const int *recvcounts, const int *displs,
                   MPI_Datatype recvtype, MPI_Comm comm);
int MPI_Gatherv(const void *sendbuf, int sendcount, MPI_Datatype sendtype,
                void *recvbuf, const int *recvcounts, const int *displs,
                MPI_Datatype recvtype, int root, MPI_Comm comm);
int MPI_Scatterv(const void *sendbuf, const int *sendcounts, const int *displs,
                 MPI_Datatype sendtype, void *recvbuf, int recvcount,
                 MPI_Datatype recvtype, int root, MPI_Comm comm);
int MPI_Wait(MPI_Request *req, MPI_Status *status);
int MPI_Waitall(int count, MPI_Request *reqs, MPI_Status *statuses);
int MPI_Isend(const void *buf, int count, MPI_Datatype type, int dest, int tag,
              MPI_Comm comm, MPI_Request *req);
int MPI_Irecv(void *buf, int count, MPI_Datatype type, int source, int tag,
              MPI_Comm comm, MPI_Request *req);
int MPI_Send(const void *buf, int count, MPI_Datatype type, int dest, int tag,
             MPI_Comm comm, ...);
int MPI_Recv(void *buf, int count, MPI_Datatype type, int source, int tag,
             MPI_Comm comm, MPI_Status *status);
int MPI_Sendrecv(const void *sendbuf, int sendcount, MPI_Datatype sendtype, int dest,
                 int sendtag, void *recvbuf, int recvcount, MPI_Datatype recvtype,
                 int source, int recvtag, MPI_Comm comm, MPI_Status *status);
int MPI_Sendrecv_replace(void *buf, int count, MPI_Datatype type, int dest,
                         int sendtag, int source, int recvtag, MPI_Comm comm,
                         MPI_Status *status);

#ifdef __cplusplus
}
#endif
#endif
