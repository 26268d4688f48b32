// gpu_shim.cpp - the reference's GPU entry points (include/gpu.hpp:35-49) over librast3d_b200.
//
// This is the reference-side binding: compiled together with the reference's own sources and
// its unmodified src/main.cpp (-DR3D_HAVE_GPU), it puts the B200 library behind the
// reference's `--backend gpu` time loop (src/main.cpp:234-275) in place of src/gpu.cpp and
// src/gpu_kernels.cu.  The functions keep the reference's names, C++ signatures and error
// behaviour (a failure prints a message and aborts the MPI job, src/gpu.cpp:117-139).
//
// The reference decomposes the domain over npey x npez MPI ranks and gives each rank a GPU.
// The library holds the whole domain on one GPU, or one z slab per GPU.  Two modes, chosen once
// per job by every rank alike:
//  * gather (every rank on the same GPU, or npey > 1): rank 0 owns one whole-domain handle.
//    gpu_upload gathers the rank blocks into the global arrays (interiors, plus the domain's
//    ghost layers from the edge ranks) and gpu_download scatters them back, halos included;
//    step_gpu steps on rank 0 and broadcasts the scalars.
//  * slabs (npey == 1, one distinct GPU per rank): each rank owns a z-slab handle over its own
//    block (r3d_gpu_create_slab) and the handles exchange ghost planes over NCCL
//    (r3d_gpu_halo_init, the id broadcast over the job's communicator); no gather.
// R3D_SHIM_MODE=gather|slabs overrides the choice.  R3D_GPU_PRECISION=fp32bulk selects the
// FP32-bulk form (default fp64: bit-exact with the CPU path).
//
// The mode is decided by the first gpu_upload (collective), from the GPU current on each rank
// (src/main.cpp:238 selects it before gpu_alloc).  gpu_alloc and gpu_upload receive no Params,
// so the library handle is created by the first step_gpu, which has them; gpu_upload stages the
// state until then.  gpu_upload and gpu_download communicate on MPI_COMM_WORLD, as src/main.cpp
// does for every collective; step_gpu uses the comm it is given.
#include <mpi.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime_api.h>
#include <unistd.h>

#include "gpu.hpp"
#include "r3d_gpu.h"

namespace r3d {

namespace {

[[noreturn]] void shim_fail(const std::string& what) {
    fprintf(stderr, "rast-3dmhd (B200 library): %s\n", what.c_str());
    fflush(stderr);
    MPI_Abort(MPI_COMM_WORLD, 1);
    std::abort();  // MPI_Abort does not return
}

void ok(int rc, const char* what) {
    if (rc != R3D_OK) shim_fail(std::string(what) + ": " + r3d_last_error());
}

// the reference Params as the library's configuration struct (same fields, same meaning)
r3d_params to_r3d(const Params& p) {
    r3d_params q;
    r3d_params_default(&q);
    q.npx = p.npx; q.npy = p.npy; q.npz = p.npz; q.npey = p.npey; q.ix = p.ix; q.iy = p.iy;
    q.ilap = p.ilap; q.ipad = p.ipad; q.ngrid = p.ngrid; q.id = p.id; q.ncol = p.ncol; q.nrow = p.nrow;
    q.ixcon = p.ixcon; q.iycon = p.iycon; q.izcon = p.izcon; q.itcon = p.itcon; q.ibcon = p.ibcon;
    q.lrot = p.lrot; q.lmag = p.lmag; q.lpot = p.lpot; q.lrem = p.lrem; q.lshr = p.lshr;
    q.ncase = p.ncase; q.ncasep = p.ncasep; q.ntotal = p.ntotal; q.nstep0 = p.nstep0;
    q.nstart = p.nstart; q.ntube = p.ntube;
    q.re = p.re; q.pr = p.pr; q.theta = p.theta; q.grav = p.grav; q.r_y = p.r_y; q.ang = p.ang;
    q.rm = p.rm; q.beta = p.beta; q.pzp = p.pzp; q.sigma = p.sigma; q.polys = p.polys; q.tp = p.tp;
    q.tc = p.tc; q.xp = p.xp; q.yp = p.yp; q.zp = p.zp; q.xmax = p.xmax; q.ymax = p.ymax;
    q.zmax = p.zmax; q.ampt = p.ampt; q.ampb = p.ampb; q.bfh = p.bfh; q.bzp = p.bzp; q.qfh = p.qfh;
    q.gamma = p.gamma; q.hh = p.hh; q.dh = p.dh; q.dv = p.dv; q.tstart = p.tstart; q.toff = p.toff;
    q.rlax = p.rlax;
    q.xx1 = p.xx1; q.xx2 = p.xx2; q.yy1 = p.yy1; q.yy2 = p.yy2; q.zz1 = p.zz1; q.zz2 = p.zz2;
    q.xa = p.xa; q.xb = p.xb; q.xc = p.xc; q.xd = p.xd; q.ya = p.ya; q.yb = p.yb; q.yc = p.yc;
    q.yd = p.yd; q.za = p.za; q.zb = p.zb; q.zc = p.zc; q.zd = p.zd;
    q.xcent = p.xcent; q.zcent = p.zcent; q.rmax = p.rmax; q.cmt = p.cmt; q.a_tube = p.a_tube;
    q.lambda = p.lambda; q.vz0 = p.vz0; q.sf = p.sf;
    q.backend = 1;
    q.gpu_id = p.gpu_id;
    const char* prec = getenv("R3D_GPU_PRECISION");
    q.precision = (prec && std::string(prec) == "fp32bulk") ? R3D_PREC_FP32BULK : R3D_PREC_FP64;
    return q;
}

// Host copy of a state in the reference layout over nx x ny x nz (a rank block or the global
// domain): the primaries, the RK accumulators and the 1D metric lines.
struct HostBlock {
    int nx = 0, ny = 0, nz = 0;
    std::vector<double> f[8];   // ru rv rw ro tt bx by bz
    std::vector<double> z[8];   // zru .. ztt, zbx zby zbz
    std::vector<double> w[8];   // uu vv ww fu fv fw fr ft: the FLUXES work arrays after a full step
    std::vector<double> lx[4], ly[4], lz[6];  // exx dxxdx d2xxdx2 ddx | wyy .. ddy | zee .. ddz rkapa dkapa
    void resize(int x, int y, int zz) {
        nx = x; ny = y; nz = zz;
        const size_t n = (size_t)x * y * zz;
        for (auto& a : f) a.assign(n, 0.0);
        for (auto& a : z) a.assign(n, 0.0);
        for (auto& a : w) a.assign(n, 0.0);
        for (auto& a : lx) a.assign(x, 0.0);
        for (auto& a : ly) a.assign(y, 0.0);
        for (auto& a : lz) a.assign(zz, 0.0);
    }
    r3d_host_state view() {
        r3d_host_state s{};
        double** o[8] = {&s.ru, &s.rv, &s.rw, &s.ro, &s.tt, &s.bx, &s.by, &s.bz};
        for (int q = 0; q < 8; ++q) *o[q] = f[q].data();
        s.exx = lx[0].data(); s.dxxdx = lx[1].data(); s.d2xxdx2 = lx[2].data(); s.ddx = lx[3].data();
        s.wyy = ly[0].data(); s.dyydy = ly[1].data(); s.d2yydy2 = ly[2].data(); s.ddy = ly[3].data();
        s.zee = lz[0].data(); s.dzzdz = lz[1].data(); s.d2zzdz2 = lz[2].data(); s.ddz = lz[3].data();
        s.rkapa = lz[4].data(); s.dkapa = lz[5].data();
        return s;
    }
};

Field* field_of(SimState& s, int q) {
    Field* f[8] = {&s.ru, &s.rv, &s.rw, &s.ro, &s.tt, &s.bx, &s.by, &s.bz};
    return f[q];
}
const Field* field_of(const SimState& s, int q) { return field_of(const_cast<SimState&>(s), q); }
Field* zfield_of(SimState& s, int q) {
    Field* f[8] = {&s.zru, &s.zrv, &s.zrw, &s.zro, &s.ztt, &s.zbx, &s.zby, &s.zbz};
    return f[q];
}

// One GpuSim's binding to the library.
struct Binding {
    Derived d{};
    bool have_state = false;   // a gpu_upload has been gathered (gather mode: on rank 0)
    HostBlock staged;          // gather mode, rank 0: the global state; slabs: this rank's block
    r3d_scalars sc{};
    r3d_gpu* h = nullptr;      // gather mode: rank 0 only; slabs: every rank
    int mode = -1;             // 0 gather, 1 slabs (decided by the first gpu_upload)
    bool dirty = false;        // staged state newer than the handle's
};

std::mutex g_mu;
std::map<const GpuSim*, Binding*> g_bind;

Binding& binding(const GpuSim& g) {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_bind.find(&g);
    if (it == g_bind.end()) shim_fail("GpuSim used before gpu_alloc");
    return *it->second;
}

int world_rank() {
    int r = 0;
    MPI_Comm_rank(MPI_COMM_WORLD, &r);
    return r;
}
int world_size() {
    int n = 1;
    MPI_Comm_size(MPI_COMM_WORLD, &n);
    return n;
}

// rank layout of src/topology.cpp (include/topology.hpp:17-18): mypey = r % npey, mypez = r / npey
void rank_xy(int r, int npey, int& mypey, int& mypez) {
    mypey = r % npey;
    mypez = r / npey;
}

// Copy between a rank block (local extents of d) and the global arrays: with `gather`, the
// block's interior plus the domain's ghost layers it holds go into the global arrays; without,
// the whole block (halos included) is read back out of them.
void block_global(const Derived& d, int mypey, int mypez, HostBlock& blk, HostBlock& glob, bool gather) {
    const int nx = d.nx, ny = d.ny, nz = d.nz, NY = glob.ny;
    for (int q = 0; q < 8; ++q) {
        if (blk.f[q].empty() || glob.f[q].empty()) continue;
        for (int kl = 0; kl < nz; ++kl) {
            const bool kin = (kl >= 1 && kl <= d.nrz) || (kl == 0 && mypez == 0) ||
                             (kl == nz - 1 && mypez == d.npez - 1);
            if (gather && !kin) continue;
            const int kg = mypez * d.nrz + kl;
            for (int jl = 0; jl < ny; ++jl) {
                const bool jin = (jl >= 1 && jl <= d.nry) || (jl == 0 && mypey == 0) ||
                                 (jl == ny - 1 && mypey == d.npey - 1);
                if (gather && !jin) continue;
                const int jg = mypey * d.nry + jl;
                double* b = blk.f[q].data() + ((size_t)kl * ny + jl) * nx;
                double* gz = glob.f[q].data() + ((size_t)kg * NY + jg) * nx;
                double* bz = blk.z[q].data() + ((size_t)kl * ny + jl) * nx;
                double* gzz = glob.z[q].data() + ((size_t)kg * NY + jg) * nx;
                double* bw = blk.w[q].data() + ((size_t)kl * ny + jl) * nx;
                double* gw = glob.w[q].data() + ((size_t)kg * NY + jg) * nx;
                if (gather) {
                    memcpy(gz, b, nx * sizeof(double));
                    memcpy(gzz, bz, nx * sizeof(double));
                    memcpy(gw, bw, nx * sizeof(double));
                } else {
                    memcpy(b, gz, nx * sizeof(double));
                    memcpy(bz, gzz, nx * sizeof(double));
                    memcpy(bw, gw, nx * sizeof(double));
                }
            }
        }
    }
    if (!gather) return;
    if (mypey == 0 && mypez == 0)  // x is not decomposed: rank 0's lines (other blocks carry none)
        for (int q = 0; q < 4; ++q) glob.lx[q] = blk.lx[q];
    if (mypez == 0)
        for (int jl = 0; jl < ny; ++jl) {
            const bool jin = (jl >= 1 && jl <= d.nry) || (jl == 0 && mypey == 0) ||
                             (jl == ny - 1 && mypey == d.npey - 1);
            if (jin)
                for (int q = 0; q < 4; ++q) glob.ly[q][mypey * d.nry + jl] = blk.ly[q][jl];
        }
    if (mypey == 0)
        for (int kl = 0; kl < nz; ++kl) {
            const bool kin = (kl >= 1 && kl <= d.nrz) || (kl == 0 && mypez == 0) ||
                             (kl == nz - 1 && mypez == d.npez - 1);
            if (kin)
                for (int q = 0; q < 6; ++q) glob.lz[q][mypez * d.nrz + kl] = blk.lz[q][kl];
        }
}

void from_state(const SimState& s, HostBlock& blk) {
    const Derived& d = s.d;
    blk.resize(d.nx, d.ny, d.nz);
    for (int q = 0; q < 8; ++q) {
        const Field* f = field_of(s, q);
        memcpy(blk.f[q].data(), f->data(), f->size() * sizeof(double));
    }
    const std::vector<double>* lx[4] = {&s.exx, &s.dxxdx, &s.d2xxdx2, &s.ddx};
    const std::vector<double>* ly[4] = {&s.wyy, &s.dyydy, &s.d2yydy2, &s.ddy};
    const std::vector<double>* lz[6] = {&s.zee, &s.dzzdz, &s.d2zzdz2, &s.ddz, &s.rkapa, &s.dkapa};
    for (int q = 0; q < 4; ++q) blk.lx[q] = *lx[q];
    for (int q = 0; q < 4; ++q) blk.ly[q] = *ly[q];
    for (int q = 0; q < 6; ++q) blk.lz[q] = *lz[q];
}

void to_state(HostBlock& blk, SimState& s) {
    Field* w[8] = {&s.uu, &s.vv, &s.ww, &s.fu, &s.fv, &s.fw, &s.fr, &s.ft};
    for (int q = 0; q < 8; ++q) {
        memcpy(field_of(s, q)->data(), blk.f[q].data(), blk.f[q].size() * sizeof(double));
        memcpy(zfield_of(s, q)->data(), blk.z[q].data(), blk.z[q].size() * sizeof(double));
        memcpy(w[q]->data(), blk.w[q].data(), blk.w[q].size() * sizeof(double));
    }
}

// A rank's FLUXES forms FU..FT on its own interior only (src/fluxes.cpp:74-76); the values a
// block cut from the global arrays carries on its halo cells are not the rank's.
void clear_flux_halo(HostBlock& blk) {
    const int nx = blk.nx, ny = blk.ny, nz = blk.nz;
    for (int q = 3; q < 8; ++q)
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i)
                    if (k == 0 || k == nz - 1 || j == 0 || j == ny - 1 || i == 0 || i == nx - 1)
                        blk.w[q][((size_t)k * ny + j) * nx + i] = 0.0;
}

// The dump's FLUXES work arrays of the handle's last full step (r3d_gpu_download_work); zeros
// when the state has not taken a full step since it was uploaded, and in the FP32-bulk form,
// which keeps no FP64 work arrays.
void fetch_work(r3d_gpu* h, HostBlock& blk) {
    std::vector<double*> w(8);
    for (int q = 0; q < 8; ++q) w[q] = blk.w[q].data();
    const int rc = r3d_gpu_download_work(h, w.data());
    if (rc == R3D_ESTATE || rc == R3D_EINVAL) {
        for (auto& a : blk.w) std::fill(a.begin(), a.end(), 0.0);
        return;
    }
    ok(rc, "r3d_gpu_download_work");
}

constexpr int kTagField = 7100;

// Send / receive the primaries and accumulators of a block, field by field.
void send_block(HostBlock& blk, int dest, bool with_z) {
    for (int q = 0; q < 8; ++q) {
        MPI_Send(blk.f[q].data(), (int)blk.f[q].size(), MPI_DOUBLE, dest, kTagField + q, MPI_COMM_WORLD);
        if (with_z) {
            MPI_Send(blk.z[q].data(), (int)blk.z[q].size(), MPI_DOUBLE, dest, kTagField + 8 + q, MPI_COMM_WORLD);
            MPI_Send(blk.w[q].data(), (int)blk.w[q].size(), MPI_DOUBLE, dest, kTagField + 30 + q, MPI_COMM_WORLD);
        }
    }
}
void recv_block(HostBlock& blk, int src, bool with_z, bool with_lines) {
    for (int q = 0; q < 8; ++q) {
        MPI_Recv(blk.f[q].data(), (int)blk.f[q].size(), MPI_DOUBLE, src, kTagField + q, MPI_COMM_WORLD,
                 MPI_STATUS_IGNORE);
        if (with_z) {
            MPI_Recv(blk.z[q].data(), (int)blk.z[q].size(), MPI_DOUBLE, src, kTagField + 8 + q, MPI_COMM_WORLD,
                     MPI_STATUS_IGNORE);
            MPI_Recv(blk.w[q].data(), (int)blk.w[q].size(), MPI_DOUBLE, src, kTagField + 30 + q, MPI_COMM_WORLD,
                     MPI_STATUS_IGNORE);
        }
    }
    if (with_lines) {
        for (auto& a : blk.ly) MPI_Recv(a.data(), (int)a.size(), MPI_DOUBLE, src, kTagField + 20, MPI_COMM_WORLD, MPI_STATUS_IGNORE);
        for (auto& a : blk.lz) MPI_Recv(a.data(), (int)a.size(), MPI_DOUBLE, src, kTagField + 21, MPI_COMM_WORLD, MPI_STATUS_IGNORE);
    }
}
void send_lines(HostBlock& blk, int dest) {
    for (auto& a : blk.ly) MPI_Send(a.data(), (int)a.size(), MPI_DOUBLE, dest, kTagField + 20, MPI_COMM_WORLD);
    for (auto& a : blk.lz) MPI_Send(a.data(), (int)a.size(), MPI_DOUBLE, dest, kTagField + 21, MPI_COMM_WORLD);
}

// 64-bit FNV-1a of this rank's GPU (host name and PCI bus id of device gpu_id)
uint64_t device_key(int gpu_id) {
    char host[256] = {0}, bus[64] = {0};
    gethostname(host, sizeof(host) - 1);
    if (cudaDeviceGetPCIBusId(bus, sizeof(bus), gpu_id) != cudaSuccess) snprintf(bus, sizeof(bus), "dev%d", gpu_id);
    uint64_t h = 1469598103934665603ull;
    const char* parts[3] = {host, ":", bus};
    for (const char* s : parts)
        for (const char* c = s; *c; ++c) h = (h ^ (unsigned char)*c) * 1099511628211ull;
    return h;
}

// gather (0) or slabs (1), the same on every rank (collective): slabs when npey == 1 and every
// rank's current GPU is its own
int choose_mode(const Derived& d) {
    const char* env = getenv("R3D_SHIM_MODE");
    if (env && std::string(env) == "gather") return 0;
    if (env && std::string(env) == "slabs") {
        if (d.npey != 1) shim_fail("R3D_SHIM_MODE=slabs needs --npey 1 (z slabs only)");
        return 1;
    }
    const int me = world_rank(), npe = world_size();
    if (d.npey != 1 || npe == 1) return 0;
    int dev = 0;
    cudaGetDevice(&dev);
    const uint64_t mine = device_key(dev);
    std::vector<uint64_t> all(npe, 0);
    for (int r = 0; r < npe; ++r) {
        uint64_t v = (r == me) ? mine : 0;
        MPI_Bcast(&v, (int)sizeof(v), MPI_BYTE, r, MPI_COMM_WORLD);
        all[r] = v;
    }
    for (int a = 0; a < npe; ++a)
        for (int b = a + 1; b < npe; ++b)
            if (all[a] == all[b]) return 0;
    return 1;
}

void scalars_from(const SimState& s, r3d_scalars& sc) {
    sc.dt = s.dt; sc.timc = s.timc; sc.timt = s.timt; sc.timi = s.timi; sc.umach = s.umach;
    sc.tb = s.tb; sc.nit = s.nit;
}
void scalars_to(const r3d_scalars& sc, SimState& s) {
    s.dt = sc.dt; s.timc = sc.timc; s.timt = sc.timt; s.umach = sc.umach; s.nit = sc.nit;
}

// Creates the handle(s) and uploads the staged state: the first step_gpu.
void ensure_handle(Binding& b, const Params& p, const Topology& t) {
    const r3d_params q = to_r3d(p);
    if (b.mode == 0) {
        if (t.mype == 0 && !b.h) ok(r3d_gpu_create(&q, &b.h), "r3d_gpu_create");
    } else if (!b.h) {
        const int nrz = p.npz / t.npez;
        ok(r3d_gpu_create_slab(&q, t.mypez * nrz, nrz, &b.h), "r3d_gpu_create_slab");
        unsigned char uid[128] = {0};
        if (t.mypez == 0) ok(r3d_nccl_unique_id(uid, sizeof(uid)), "r3d_nccl_unique_id");
        MPI_Bcast(uid, (int)sizeof(uid), MPI_BYTE, 0, MPI_COMM_WORLD);
        ok(r3d_gpu_halo_init(b.h, uid, sizeof(uid), t.mypez, t.npez), "r3d_gpu_halo_init");
    }
    if (b.h && b.dirty) {
        r3d_host_state v = b.staged.view();
        ok(r3d_gpu_upload(b.h, &v, &b.sc), "r3d_gpu_upload");
        b.dirty = false;
    }
}

}  // namespace

void gpu_alloc(GpuSim& g, const Derived& d) {
    auto* b = new Binding();
    b->d = d;
    g.nx = d.nx;
    g.ny = d.ny;
    g.nz = d.nz;
    std::lock_guard<std::mutex> lk(g_mu);
    g_bind[&g] = b;
}

void gpu_upload(GpuSim& g, const SimState& s) {
    Binding& b = binding(g);
    const Derived& d = b.d;
    const int me = world_rank(), npe = world_size();
    scalars_from(s, b.sc);
    HostBlock mine;
    from_state(s, mine);
    if (b.mode < 0) b.mode = choose_mode(d);
    if (b.mode == 1) {  // slabs: every rank uploads its own block
        b.staged = std::move(mine);
        b.dirty = true;
        if (b.h) {
            r3d_host_state v = b.staged.view();
            ok(r3d_gpu_upload(b.h, &v, &b.sc), "r3d_gpu_upload");
            b.dirty = false;
        }
        b.have_state = true;
        return;
    }
    // gather mode: rank 0 assembles the global state
    if (me == 0) {
        HostBlock glob;
        glob.resize(d.nx, d.npey * d.nry + 2, d.npez * d.nrz + 2);
        for (int r = 0; r < npe; ++r) {
            int py, pz;
            rank_xy(r, d.npey, py, pz);
            HostBlock blk;
            if (r == 0) {
                blk = mine;
            } else {
                blk.resize(d.nx, d.ny, d.nz);
                recv_block(blk, r, false, true);
            }
            block_global(d, py, pz, blk, glob, true);
        }
        b.staged = std::move(glob);
    } else {
        send_block(mine, 0, false);
        send_lines(mine, 0);
    }
    b.have_state = true;
    b.dirty = true;
    if (b.h) {  // a handle exists already (a re-upload): refresh it now
        r3d_host_state v = b.staged.view();
        ok(r3d_gpu_upload(b.h, &v, &b.sc), "r3d_gpu_upload");
        b.dirty = false;
    }
}

void gpu_download(SimState& s, GpuSim& g) {
    Binding& b = binding(g);
    const Derived& d = b.d;
    const int me = world_rank(), npe = world_size();
    if (!b.have_state) shim_fail("gpu_download before gpu_upload");
    if (b.mode == 1) {
        if (b.h && !b.dirty) {
            r3d_host_state v = b.staged.view();
            ok(r3d_gpu_download(b.h, &v, &b.sc), "r3d_gpu_download");
            std::vector<double*> z(8, nullptr);
            for (int q = 0; q < 8; ++q) z[q] = b.staged.z[q].data();
            ok(r3d_gpu_download_accumulators(b.h, z.data()), "r3d_gpu_download_accumulators");
            fetch_work(b.h, b.staged);
        }
        to_state(b.staged, s);
        scalars_to(b.sc, s);
        return;
    }
    if (me == 0) {
        if (b.h && !b.dirty) {
            r3d_host_state v = b.staged.view();
            ok(r3d_gpu_download(b.h, &v, &b.sc), "r3d_gpu_download");
            std::vector<double*> z(8, nullptr);
            for (int q = 0; q < 8; ++q) z[q] = b.staged.z[q].data();
            ok(r3d_gpu_download_accumulators(b.h, z.data()), "r3d_gpu_download_accumulators");
            fetch_work(b.h, b.staged);
        }
        for (int r = npe - 1; r >= 0; --r) {
            int py, pz;
            rank_xy(r, d.npey, py, pz);
            HostBlock blk;
            blk.resize(d.nx, d.ny, d.nz);
            block_global(d, py, pz, blk, b.staged, false);
            clear_flux_halo(blk);
            if (r == 0) to_state(blk, s);
            else send_block(blk, r, true);
        }
    } else {
        HostBlock blk;
        blk.resize(d.nx, d.ny, d.nz);
        recv_block(blk, 0, true, false);
        to_state(blk, s);
    }
    double v[5] = {b.sc.dt, b.sc.timc, b.sc.timt, b.sc.umach, (double)b.sc.nit};
    MPI_Bcast(v, 5, MPI_DOUBLE, 0, MPI_COMM_WORLD);
    b.sc.dt = v[0]; b.sc.timc = v[1]; b.sc.timt = v[2]; b.sc.umach = v[3]; b.sc.nit = (int)v[4];
    scalars_to(b.sc, s);
}

void gpu_free(GpuSim& g) {
    Binding* b = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        auto it = g_bind.find(&g);
        if (it == g_bind.end()) return;
        b = it->second;
        g_bind.erase(it);
    }
    if (b->h) r3d_gpu_destroy(b->h);
    delete b;
}

void step_gpu(int nstages, MPI_Comm comm, const Params& p, const Derived& d, const Topology& t, GpuSim& g,
              SimState& scalars) {
    (void)d;
    Binding& b = binding(g);
    if (!b.have_state) shim_fail("step_gpu before gpu_upload");
    ensure_handle(b, p, t);
    if (b.mode == 1) {
        ok(r3d_gpu_step(b.h, nstages, &b.sc), "r3d_gpu_step");
        scalars_to(b.sc, scalars);
        return;
    }
    double v[5] = {0, 0, 0, 0, 0};
    if (t.mype == 0) {
        const int rc = r3d_gpu_step(b.h, nstages, &b.sc);
        v[4] = rc == R3D_OK ? (double)b.sc.nit : -1.0;
        v[0] = b.sc.dt; v[1] = b.sc.timc; v[2] = b.sc.timt; v[3] = b.sc.umach;
        if (rc != R3D_OK) fprintf(stderr, "rast-3dmhd (B200 library): r3d_gpu_step: %s\n", r3d_last_error());
    }
    MPI_Bcast(v, 5, MPI_DOUBLE, 0, comm);
    if (v[4] < 0) shim_fail("r3d_gpu_step failed on rank 0");
    b.sc.dt = v[0]; b.sc.timc = v[1]; b.sc.timt = v[2]; b.sc.umach = v[3]; b.sc.nit = (int)v[4];
    scalars_to(b.sc, scalars);
}

void step_gpu(MPI_Comm comm, const Params& p, const Derived& d, const Topology& t, GpuSim& g,
              SimState& scalars) {
    step_gpu(3, comm, p, d, t, g, scalars);
}

}  // namespace r3d
