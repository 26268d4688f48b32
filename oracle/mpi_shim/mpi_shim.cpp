// Thread-rank MPI stand-in: in-process mailboxes and a slot-table for collectives.
//
// Test infrastructure only (see mpi.h).  Sends are buffered (the payload is copied into the
// destination's mailbox and the call returns), so the reference's Send/Recv orderings in
// src/communicate.cpp:81-156 and src/static_ic.cpp:122-153 cannot deadlock.  Collectives
// use a generation-counted barrier; MIN/MAX are exact, so the reduction order is irrelevant.
// MPI_Abort marks the world aborted and throws; every blocked call then throws as well, so a
// failing rank cannot leave the others waiting forever.
#include "mpi.h"

#include <algorithm>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <stdexcept>
#include <tuple>
#include <vector>

namespace {

struct World {
    std::mutex mu;
    std::condition_variable cv;
    int nranks = 1;
    bool aborted = false;
    // (src, dst, tag) -> FIFO of payloads
    std::map<std::tuple<int, int, int>, std::deque<std::vector<char>>> box;
    // collective slots
    std::vector<std::vector<char>> slot;
    int arrived = 0;
    long generation = 0;
};

World g_world;
thread_local int t_rank = 0;

size_t type_size(MPI_Datatype t) {
    switch (t) {
        case MPI_DOUBLE: return sizeof(double);
        case MPI_BYTE: return 1;
        case MPI_INT: return sizeof(int);
        default: throw std::runtime_error("mpi shim: unsupported datatype");
    }
}

void check_abort_locked() {
    if (g_world.aborted) throw std::runtime_error("mpi shim: world aborted");
}

// Barrier over all ranks; must be called with the lock held.
void barrier_locked(std::unique_lock<std::mutex>& lk) {
    long gen = g_world.generation;
    if (++g_world.arrived == g_world.nranks) {
        g_world.arrived = 0;
        ++g_world.generation;
        g_world.cv.notify_all();
        return;
    }
    g_world.cv.wait(lk, [&] { return g_world.generation != gen || g_world.aborted; });
    check_abort_locked();
}

}  // namespace

extern "C" {

void r3d_shim_world_init(int nranks) {
    std::lock_guard<std::mutex> lk(g_world.mu);
    g_world.nranks = nranks;
    g_world.aborted = false;
    g_world.box.clear();
    g_world.slot.assign(nranks, {});
    g_world.arrived = 0;
}

void r3d_shim_bind_rank(int rank) { t_rank = rank; }

int MPI_Init(int*, char***) { return MPI_SUCCESS; }
int MPI_Finalize(void) { return MPI_SUCCESS; }

int MPI_Comm_size(MPI_Comm, int* size) {
    *size = g_world.nranks;
    return MPI_SUCCESS;
}

int MPI_Comm_rank(MPI_Comm, int* rank) {
    *rank = t_rank;
    return MPI_SUCCESS;
}

int MPI_Send(const void* buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm) {
    size_t n = (size_t)count * type_size(type);
    std::vector<char> payload(n);
    if (n) std::memcpy(payload.data(), buf, n);
    std::lock_guard<std::mutex> lk(g_world.mu);
    check_abort_locked();
    g_world.box[std::make_tuple(t_rank, dest, tag)].push_back(std::move(payload));
    g_world.cv.notify_all();
    return MPI_SUCCESS;
}

int MPI_Recv(void* buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm,
             MPI_Status* status) {
    size_t n = (size_t)count * type_size(type);
    std::unique_lock<std::mutex> lk(g_world.mu);
    auto key = std::make_tuple(source, t_rank, tag);
    g_world.cv.wait(lk, [&] {
        if (g_world.aborted) return true;
        auto it = g_world.box.find(key);
        return it != g_world.box.end() && !it->second.empty();
    });
    check_abort_locked();
    auto& q = g_world.box[key];
    std::vector<char> payload = std::move(q.front());
    q.pop_front();
    if (payload.size() > n) throw std::runtime_error("mpi shim: message truncated");
    if (!payload.empty()) std::memcpy(buf, payload.data(), payload.size());
    if (status) {
        status->MPI_SOURCE = source;
        status->MPI_TAG = tag;
        status->MPI_ERROR = 0;
    }
    return MPI_SUCCESS;
}

int MPI_Sendrecv(const void* sendbuf, int sendcount, MPI_Datatype sendtype, int dest, int sendtag,
                 void* recvbuf, int recvcount, MPI_Datatype recvtype, int source, int recvtag,
                 MPI_Comm comm, MPI_Status* status) {
    MPI_Send(sendbuf, sendcount, sendtype, dest, sendtag, comm);
    return MPI_Recv(recvbuf, recvcount, recvtype, source, recvtag, comm, status);
}

int MPI_Allreduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype type, MPI_Op op,
                  MPI_Comm) {
    size_t n = (size_t)count * type_size(type);
    std::unique_lock<std::mutex> lk(g_world.mu);
    check_abort_locked();
    g_world.slot[t_rank].assign((const char*)sendbuf, (const char*)sendbuf + n);
    barrier_locked(lk);
    if (type != MPI_DOUBLE) throw std::runtime_error("mpi shim: Allreduce supports doubles only");
    std::vector<double> acc(count);
    std::memcpy(acc.data(), g_world.slot[0].data(), n);
    for (int r = 1; r < g_world.nranks; ++r) {
        const double* v = (const double*)g_world.slot[r].data();
        for (int i = 0; i < count; ++i) {
            if (op == MPI_MIN)
                acc[i] = std::min(acc[i], v[i]);
            else if (op == MPI_MAX)
                acc[i] = std::max(acc[i], v[i]);
            else
                acc[i] = acc[i] + v[i];
        }
    }
    std::memcpy(recvbuf, acc.data(), n);
    barrier_locked(lk);  // slots may be reused only after every rank has read them
    return MPI_SUCCESS;
}

int MPI_Bcast(void* buf, int count, MPI_Datatype type, int root, MPI_Comm) {
    size_t n = (size_t)count * type_size(type);
    std::unique_lock<std::mutex> lk(g_world.mu);
    check_abort_locked();
    if (t_rank == root) g_world.slot[root].assign((const char*)buf, (const char*)buf + n);
    barrier_locked(lk);
    if (t_rank != root) std::memcpy(buf, g_world.slot[root].data(), n);
    barrier_locked(lk);
    return MPI_SUCCESS;
}

int MPI_Abort(MPI_Comm, int errorcode) {
    {
        std::lock_guard<std::mutex> lk(g_world.mu);
        g_world.aborted = true;
        g_world.cv.notify_all();
    }
    char msg[64];
    std::snprintf(msg, sizeof(msg), "mpi shim: MPI_Abort(%d)", errorcode);
    throw std::runtime_error(msg);
}

}  // extern "C"
