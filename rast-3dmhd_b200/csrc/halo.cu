// halo.cu - z-slab decomposition across processes: ghost-plane exchange and the dt reduction
// over NCCL (one process per GPU).
//
// The reference splits the domain over npey x npez MPI ranks and, after every stage, exchanges
// one ghost plane per face with MPI or NCCL (src/communicate.cpp:70-182), plus one MPI_Allreduce
// (min) of the time-step limits per step (src/step.cpp:224).  Here each process holds one z slab
// (r3d_gpu_create_slab) on its own GPU; after every stage its first and last planes go to the z
// neighbours' ghost planes with ncclSend/ncclRecv (whole contiguous planes, ghost columns
// included, every field of the state), and before every step the four limit minima and the Mach
// maximum, kept on the device as ordered-integer keys, are combined with ncclAllReduce (uint64
// min / max).  Everything is queued on the library's stream: no host round trip.  The keys make
// the reduction exact and order-free, so every slab count gives the bit-identical dt of the
// single-domain run.
//
// NCCL is loaded at run time, so the library itself has no link-time NCCL dependency: an NCCL
// the process has already loaded (a PyTorch process has its own) is used as it is; otherwise
// $R3D_NCCL_LIBRARY or libnccl.so.2 is opened with local symbol scope, so that a later import of
// PyTorch still binds to its own NCCL.
#include <dlfcn.h>
#include <nccl.h>

#include <cstdlib>
#include <cstring>
#include <string>

#include "r3d_gpu_impl.hpp"

using namespace r3db;

namespace r3dg {

struct Nccl {
    void* dl = nullptr;
    decltype(&ncclGetUniqueId) getUniqueId = nullptr;
    decltype(&ncclCommInitRank) commInitRank = nullptr;
    decltype(&ncclCommDestroy) commDestroy = nullptr;
    decltype(&ncclSend) send = nullptr;
    decltype(&ncclRecv) recv = nullptr;
    decltype(&ncclAllReduce) allReduce = nullptr;
    decltype(&ncclGroupStart) groupStart = nullptr;
    decltype(&ncclGroupEnd) groupEnd = nullptr;
    decltype(&ncclGetErrorString) errorString = nullptr;
};

struct Halo {
    ncclComm_t comm = nullptr;
    int rank = 0, nranks = 1;
};

namespace {

Nccl& nccl() {
    static Nccl n;
    if (n.dl) return n;
    void* dl = dlopen("libnccl.so.2", RTLD_NOW | RTLD_NOLOAD);
    if (!dl) {
        const char* path = std::getenv("R3D_NCCL_LIBRARY");
        dl = dlopen(path && *path ? path : "libnccl.so.2", RTLD_NOW | RTLD_LOCAL);
    }
    if (!dl) throw Error(R3D_EINVAL, std::string("NCCL is not available: ") + dlerror());
    auto sym = [&](const char* name) {
        void* f = dlsym(dl, name);
        if (!f) throw Error(R3D_EINVAL, std::string("NCCL symbol missing: ") + name);
        return f;
    };
    n.getUniqueId = (decltype(n.getUniqueId))sym("ncclGetUniqueId");
    n.commInitRank = (decltype(n.commInitRank))sym("ncclCommInitRank");
    n.commDestroy = (decltype(n.commDestroy))sym("ncclCommDestroy");
    n.send = (decltype(n.send))sym("ncclSend");
    n.recv = (decltype(n.recv))sym("ncclRecv");
    n.allReduce = (decltype(n.allReduce))sym("ncclAllReduce");
    n.groupStart = (decltype(n.groupStart))sym("ncclGroupStart");
    n.groupEnd = (decltype(n.groupEnd))sym("ncclGroupEnd");
    n.errorString = (decltype(n.errorString))sym("ncclGetErrorString");
    n.dl = dl;
    return n;
}

void nccl_ok(ncclResult_t r, const char* what) {
    if (r != ncclSuccess) throw Error(R3D_ECUDA, std::string(what) + ": " + nccl().errorString(r));
}

}  // namespace

void halo_free(r3d_gpu* g) {
    if (!g->halo) return;
    if (g->halo->comm) nccl().commDestroy(g->halo->comm);
    delete g->halo;
    g->halo = nullptr;
}

void halo_reduce_limits(r3d_gpu* g) {
    Range r("r3d.halo_reduce");
    Halo* h = g->halo;
    Nccl& n = nccl();
    cuda_ok(r3dk::launch_save_local_limits(g->dsc, g->stream), "save local limits");
    nccl_ok(n.groupStart(), "ncclGroupStart");
    nccl_ok(n.allReduce(g->dsc->wmin, g->dsc->wmin, 4, ncclUint64, ncclMin, h->comm, g->stream), "ncclAllReduce(min)");
    nccl_ok(n.allReduce(&g->dsc->umax, &g->dsc->umax, 1, ncclUint64, ncclMax, h->comm, g->stream), "ncclAllReduce(max)");
    nccl_ok(n.groupEnd(), "ncclGroupEnd");
}

void halo_exchange(r3d_gpu* g) {
    Range r("r3d.halo_exchange");
    Halo* h = g->halo;
    Nccl& n = nccl();
    const size_t plane = (size_t)g->geo.plane;
    const int nf = state_fields(g);
    nccl_ok(n.groupStart(), "ncclGroupStart");
    for (int q = 0; q < nf; ++q) {
        size_t es = 0;
        unsigned char* f = static_cast<unsigned char*>(state_field(g, q, &es));
        const size_t bytes = plane * es;
        if (h->rank > 0) {  // the slab above: my plane 1 -> its ghost plane; its last plane -> my plane 0
            nccl_ok(n.send(f + 1 * bytes, bytes, ncclUint8, h->rank - 1, h->comm, g->stream), "ncclSend");
            nccl_ok(n.recv(f + 0 * bytes, bytes, ncclUint8, h->rank - 1, h->comm, g->stream), "ncclRecv");
        }
        if (h->rank < h->nranks - 1) {  // the slab below
            nccl_ok(n.send(f + (size_t)g->nloc * bytes, bytes, ncclUint8, h->rank + 1, h->comm, g->stream), "ncclSend");
            nccl_ok(n.recv(f + (size_t)(g->nloc + 1) * bytes, bytes, ncclUint8, h->rank + 1, h->comm, g->stream),
                    "ncclRecv");
        }
    }
    nccl_ok(n.groupEnd(), "ncclGroupEnd");
}

}  // namespace r3dg

using namespace r3dg;

extern "C" {

int r3d_nccl_unique_id(unsigned char* out, size_t len) {
    return guarded([&] {
        if (!out || len < sizeof(ncclUniqueId)) throw std::invalid_argument("need a 128-byte buffer");
        ncclUniqueId id;
        nccl_ok(nccl().getUniqueId(&id), "ncclGetUniqueId");
        std::memcpy(out, &id, sizeof id);
    });
}

int r3d_gpu_halo_init(r3d_gpu* g, const unsigned char* id, size_t len, int rank, int nranks) {
    return guarded([&] {
        if (!g || !id || len < sizeof(ncclUniqueId)) throw std::invalid_argument("bad argument");
        if (nranks < 1 || rank < 0 || rank >= nranks) throw std::invalid_argument("bad rank / nranks");
        if ((rank == 0) != (g->z0 == 0) || (rank == nranks - 1) != (g->z0 + g->nloc == g->p.npz))
            throw std::invalid_argument("rank order must follow the z order of the slabs");
        if (g->halo) throw Error(R3D_ESTATE, "halo already initialised");
        DeviceGuard dg(g->device);
        ncclUniqueId uid;
        std::memcpy(&uid, id, sizeof uid);
        auto h = new Halo();
        h->rank = rank;
        h->nranks = nranks;
        ncclResult_t r = nccl().commInitRank(&h->comm, nranks, uid, rank);
        if (r != ncclSuccess) {
            delete h;
            nccl_ok(r, "ncclCommInitRank");
        }
        g->halo = h;
    });
}

}  // extern "C"
