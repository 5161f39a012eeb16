/*
 * Size-1 MPI shim implementation (test infrastructure for the CPU oracle).
 * With one process every collective is the identity map from the send buffer
 * to this rank's slot of the receive buffer.
 */
#include "mpi.h"

#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

static size_t type_size(MPI_Datatype t) { return (size_t)(t & 0xff); }

static void copy_if_distinct(const void *src, void *dst, size_t n_bytes) {
    if (src == MPI_IN_PLACE || src == dst || n_bytes == 0) return;
    memmove(dst, src, n_bytes);
}

static int p2p_unreachable(const char *what) {
    fprintf(stderr, "mpi shim: %s reached in a world of size 1\n", what);
    abort();
    return 1;
}

int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return MPI_SUCCESS; }
int MPI_Init_thread(int *argc, char ***argv, int required, int *provided) {
    (void)argc; (void)argv;
    if (provided) *provided = required;
    return MPI_SUCCESS;
}
int MPI_Finalize(void) { return MPI_SUCCESS; }
int MPI_Abort(MPI_Comm comm, int code) { (void)comm; exit(code); }
int MPI_Comm_rank(MPI_Comm comm, int *rank) { (void)comm; *rank = 0; return MPI_SUCCESS; }
int MPI_Comm_size(MPI_Comm comm, int *size) { (void)comm; *size = 1; return MPI_SUCCESS; }
int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm *newcomm) {
    (void)color; (void)key;
    *newcomm = comm;
    return MPI_SUCCESS;
}
double MPI_Wtime(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}
int MPI_Barrier(MPI_Comm comm) { (void)comm; return MPI_SUCCESS; }
int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root, MPI_Comm comm) {
    (void)buf; (void)count; (void)type; (void)root; (void)comm;
    return MPI_SUCCESS;
}
int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype type,
                  MPI_Op op, MPI_Comm comm) {
    (void)op; (void)comm;
    copy_if_distinct(sendbuf, recvbuf, (size_t)count * type_size(type));
    return MPI_SUCCESS;
}
int MPI_Iallreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype type,
                   MPI_Op op, MPI_Comm comm, MPI_Request *req) {
    if (req) *req = MPI_REQUEST_NULL;
    return MPI_Allreduce(sendbuf, recvbuf, count, type, op, comm);
}
int MPI_Reduce_scatter(const void *sendbuf, void *recvbuf, const int *recvcounts,
                       MPI_Datatype type, MPI_Op op, MPI_Comm comm) {
    (void)op; (void)comm;
    copy_if_distinct(sendbuf, recvbuf, (size_t)recvcounts[0] * type_size(type));
    return MPI_SUCCESS;
}
int MPI_Allgather(const void *sendbuf, int sendcount, MPI_Datatype sendtype,
                  void *recvbuf, int recvcount, MPI_Datatype recvtype, MPI_Comm comm) {
    (void)recvcount; (void)recvtype; (void)comm;
    copy_if_distinct(sendbuf, recvbuf, (size_t)sendcount * type_size(sendtype));
    return MPI_SUCCESS;
}
int MPI_Allgatherv(const void *sendbuf, int sendcount, MPI_Datatype sendtype,
                   void *recvbuf, const int *recvcounts, const int *displs,
                   MPI_Datatype recvtype, MPI_Comm comm) {
    (void)recvcounts; (void)comm;
    char *dst = (char *)recvbuf + (size_t)displs[0] * type_size(recvtype);
    copy_if_distinct(sendbuf, dst, (size_t)sendcount * type_size(sendtype));
    return MPI_SUCCESS;
}
int MPI_Gatherv(const void *sendbuf, int sendcount, MPI_Datatype sendtype,
                void *recvbuf, const int *recvcounts, const int *displs,
                MPI_Datatype recvtype, int root, MPI_Comm comm) {
    (void)recvcounts; (void)root; (void)comm;
    if (!recvbuf) return MPI_SUCCESS;
    char *dst = (char *)recvbuf + (size_t)displs[0] * type_size(recvtype);
    copy_if_distinct(sendbuf, dst, (size_t)sendcount * type_size(sendtype));
    return MPI_SUCCESS;
}
int MPI_Scatterv(const void *sendbuf, const int *sendcounts, const int *displs,
                 MPI_Datatype sendtype, void *recvbuf, int recvcount,
                 MPI_Datatype recvtype, int root, MPI_Comm comm) {
    (void)sendcounts; (void)root; (void)comm;
    if (!sendbuf) return MPI_SUCCESS;
    const char *src = (const char *)sendbuf + (size_t)displs[0] * type_size(sendtype);
    copy_if_distinct(src, recvbuf, (size_t)recvcount * type_size(recvtype));
    return MPI_SUCCESS;
}
int MPI_Wait(MPI_Request *req, MPI_Status *status) { (void)req; (void)status; return MPI_SUCCESS; }
int MPI_Waitall(int count, MPI_Request *reqs, MPI_Status *statuses) {
    (void)count; (void)reqs; (void)statuses;
    return MPI_SUCCESS;
}
int MPI_Isend(const void *buf, int count, MPI_Datatype type, int dest, int tag,
              MPI_Comm comm, MPI_Request *req) {
    (void)buf; (void)count; (void)type; (void)dest; (void)tag; (void)comm; (void)req;
    return p2p_unreachable("MPI_Isend");
}
int MPI_Irecv(void *buf, int count, MPI_Datatype type, int source, int tag,
              MPI_Comm comm, MPI_Request *req) {
    (void)buf; (void)count; (void)type; (void)source; (void)tag; (void)comm; (void)req;
    return p2p_unreachable("MPI_Irecv");
}
int MPI_Send(const void *buf, int count, MPI_Datatype type, int dest, int tag,
             MPI_Comm comm, ...) {
    (void)buf; (void)count; (void)type; (void)dest; (void)tag; (void)comm;
    return p2p_unreachable("MPI_Send");
}
int MPI_Recv(void *buf, int count, MPI_Datatype type, int source, int tag,
             MPI_Comm comm, MPI_Status *status) {
    (void)buf; (void)count; (void)type; (void)source; (void)tag; (void)comm; (void)status;
    return p2p_unreachable("MPI_Recv");
}
int MPI_Sendrecv(const void *sendbuf, int sendcount, MPI_Datatype sendtype, int dest,
                 int sendtag, void *recvbuf, int recvcount, MPI_Datatype recvtype,
                 int source, int recvtag, MPI_Comm comm, MPI_Status *status) {
    (void)dest; (void)sendtag; (void)recvcount; (void)recvtype; (void)source;
    (void)recvtag; (void)comm; (void)status;
    copy_if_distinct(sendbuf, recvbuf, (size_t)sendcount * type_size(sendtype));
    return MPI_SUCCESS;
}
int MPI_Sendrecv_replace(void *buf, int count, MPI_Datatype type, int dest,
                         int sendtag, int source, int recvtag, MPI_Comm comm,
                         MPI_Status *status) {
    (void)buf; (void)count; (void)type; (void)dest; (void)sendtag; (void)source;
    (void)recvtag; (void)comm; (void)status;
    return MPI_SUCCESS;
}
