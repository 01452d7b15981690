// mpi_shim.cpp -- in-process thread implementation of the MPI subset declared in mpi.h.
// TEST INFRASTRUCTURE: used only to build the unmodified reference as the parity oracle.
#include "mpi.h"

#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <mutex>
#include <vector>

namespace {

struct Message {
    int src, dst, tag;
    std::vector<char> data;
};

std::mutex g_mu;
std::condition_variable g_cv;
std::deque<Message> g_queue;
int g_size = 1;
thread_local int t_rank = 0;

// generation barrier
int g_bar_count = 0;
long g_bar_gen = 0;

// per-rank slots for collectives
std::vector<std::vector<char>> g_slots;

std::size_t type_size(MPI_Datatype t) { return t == MPI_INT ? sizeof(int) : sizeof(double); }

void barrier()
{
    std::unique_lock<std::mutex> lk(g_mu);
    const long gen = g_bar_gen;
    if (++g_bar_count == g_size) {
        g_bar_count = 0;
        g_bar_gen++;
        g_cv.notify_all();
    } else {
        g_cv.wait(lk, [&] { return g_bar_gen != gen; });
    }
}

void post(const void *buf, std::size_t bytes, int dst, int tag)
{
    Message m;
    m.src = t_rank;
    m.dst = dst;
    m.tag = tag;
    m.data.assign((const char *)buf, (const char *)buf + bytes);
    {
        std::lock_guard<std::mutex> lk(g_mu);
        g_queue.push_back(std::move(m));
    }
    g_cv.notify_all();
}

void take(void *buf, std::size_t bytes, int src, int tag)
{
    std::unique_lock<std::mutex> lk(g_mu);
    for (;;) {
        for (auto it = g_queue.begin(); it != g_queue.end(); ++it) {
            if (it->dst == t_rank && it->src == src && it->tag == tag) {
                if (it->data.size() != bytes) {
                    std::fprintf(stderr, "mpi shim: message size mismatch (%zu vs %zu)\n", it->data.size(), bytes);
                    std::abort();
                }
                std::memcpy(buf, it->data.data(), bytes);
                g_queue.erase(it);
                return;
            }
        }
        g_cv.wait(lk);
    }
}

template <typename T> void reduce_into(T *out, int count, MPI_Op op)
{
    for (int k = 0; k < count; k++) {
        T acc = ((const T *)g_slots[0].data())[k];
        for (int r = 1; r < g_size; r++) {
            const T x = ((const T *)g_slots[r].data())[k];
            if (op == MPI_SUM) acc += x;
            else if (op == MPI_MIN) acc = x < acc ? x : acc;
            else acc = x > acc ? x : acc;
        }
        out[k] = acc;
    }
}

} // namespace

void wenofv_shim_set_rank(int rank) { t_rank = rank; }
void wenofv_shim_set_size(int size)
{
    g_size = size;
    g_slots.assign(size, std::vector<char>());
}

int MPI_Init(int *, char ***) { return MPI_SUCCESS; }
int MPI_Finalize(void) { return MPI_SUCCESS; }
int MPI_Abort(MPI_Comm, int code)
{
    std::fprintf(stderr, "mpi shim: MPI_Abort(%d)\n", code);
    std::exit(code ? code : 1);
}
int MPI_Comm_rank(MPI_Comm, int *rank) { *rank = t_rank; return MPI_SUCCESS; }
int MPI_Comm_size(MPI_Comm, int *size) { *size = g_size; return MPI_SUCCESS; }
int MPI_Barrier(MPI_Comm) { barrier(); return MPI_SUCCESS; }

int MPI_Isend(const void *buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm, MPI_Request *req)
{
    post(buf, count * type_size(type), dest, tag);
    req->pending_recv = 0;
    return MPI_SUCCESS;
}
int MPI_Irecv(void *buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm, MPI_Request *req)
{
    req->pending_recv = 1;
    req->buf = buf;
    req->bytes = count * type_size(type);
    req->peer = source;
    req->tag = tag;
    return MPI_SUCCESS;
}
int MPI_Waitall(int count, MPI_Request *reqs, MPI_Status *statuses)
{
    for (int k = 0; k < count; k++) {
        if (reqs[k].pending_recv) {
            take(reqs[k].buf, reqs[k].bytes, reqs[k].peer, reqs[k].tag);
            reqs[k].pending_recv = 0;
            if (statuses) {
                statuses[k].MPI_SOURCE = reqs[k].peer;
                statuses[k].MPI_TAG = reqs[k].tag;
                statuses[k].MPI_ERROR = 0;
            }
        }
    }
    return MPI_SUCCESS;
}
int MPI_Send(const void *buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm)
{
    post(buf, count * type_size(type), dest, tag);
    return MPI_SUCCESS;
}
int MPI_Recv(void *buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm, MPI_Status *status)
{
    take(buf, count * type_size(type), source, tag);
    if (status) {
        status->MPI_SOURCE = source;
        status->MPI_TAG = tag;
        status->MPI_ERROR = 0;
    }
    return MPI_SUCCESS;
}
int MPI_Reduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype type, MPI_Op op, int root, MPI_Comm)
{
    const std::size_t bytes = count * type_size(type);
    barrier();
    g_slots[t_rank].assign((const char *)sendbuf, (const char *)sendbuf + bytes);
    barrier();
    if (t_rank == root) {
        if (type == MPI_INT) reduce_into((int *)recvbuf, count, op);
        else reduce_into((double *)recvbuf, count, op);
    }
    barrier();
    return MPI_SUCCESS;
}
int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype type, MPI_Op op, MPI_Comm)
{
    const std::size_t bytes = count * type_size(type);
    barrier();
    g_slots[t_rank].assign((const char *)sendbuf, (const char *)sendbuf + bytes);
    barrier();
    if (type == MPI_INT) reduce_into((int *)recvbuf, count, op);
    else reduce_into((double *)recvbuf, count, op);
    barrier();
    return MPI_SUCCESS;
}
int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root, MPI_Comm)
{
    const std::size_t bytes = count * type_size(type);
    barrier();
    if (t_rank == root) g_slots[root].assign((const char *)buf, (const char *)buf + bytes);
    barrier();
    if (t_rank != root) std::memcpy(buf, g_slots[root].data(), bytes);
    barrier();
    return MPI_SUCCESS;
}
