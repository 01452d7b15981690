// mpi.h -- minimal in-process MPI shim used ONLY to build the unmodified reference
// solver (src/WENOFV.cpp, src/main.cpp) as the parity oracle and the CPU baseline.
//
// TEST INFRASTRUCTURE.  Ranks are threads of one process (the harness starts them);
// messages are buffered copies matched by (source, destination, tag) in FIFO order,
// which is the MPI non-overtaking rule.  Only the calls the reference makes exist:
// Init/Finalize/Abort, Comm_rank/size, Barrier, Isend/Irecv/Waitall, Send/Recv,
// Allreduce, Reduce, Bcast with MPI_INT/MPI_DOUBLE and SUM/MIN/MAX.
#ifndef WENOFV_MPI_SHIM_H
#define WENOFV_MPI_SHIM_H
#include <cstddef>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
#define MPI_COMM_WORLD 0
#define MPI_INT 1
#define MPI_DOUBLE 2
#define MPI_SUM 1
#define MPI_MIN 2
#define MPI_MAX 3
#define MPI_SUCCESS 0

struct MPI_Status {
    int MPI_SOURCE;
    int MPI_TAG;
    int MPI_ERROR;
};
struct MPI_Request {
    int pending_recv;
    void *buf;
    std::size_t bytes;
    int peer;
    int tag;
};
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Abort(MPI_Comm comm, int code);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Barrier(MPI_Comm comm);
int MPI_Isend(const void *buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm, MPI_Request *req);
int MPI_Irecv(void *buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm comm, MPI_Request *req);
int MPI_Waitall(int count, MPI_Request *reqs, MPI_Status *statuses);
int MPI_Send(const void *buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm);
int MPI_Recv(void *buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm comm, MPI_Status *status);
int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype type, MPI_Op op, MPI_Comm comm);
int MPI_Reduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype type, MPI_Op op, int root, MPI_Comm comm);
int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root, MPI_Comm comm);

// harness side: the rank of the calling thread and the world size
void wenofv_shim_set_rank(int rank);
void wenofv_shim_set_size(int size);

#endif
