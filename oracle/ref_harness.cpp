// Oracle harness around the reference's own CPU implementation (test infrastructure only).
//
// Links the reference sources src/{params,topology,grid,ode,ran2,static_ic,fluxes,bcon,step,
// communicate}.cpp, compiled unmodified by oracle/Makefile, against the thread-rank MPI shim.
// It reproduces the set-up sequence of the reference driver (src/main.cpp:125-154: parse_args
// -> resolve_topology -> derive -> build_grid_metrics -> rkapa/dkapa -> static_ic ->
// communicate), runs `step` (src/step.cpp:114-261) on every thread-rank, and stitches the
// rank-local blocks back into one global (npx+2) x (npy+2) x (npz+2) x-fastest array.
//
// Seeds: the reference hard-wires the RAN2 seed idum = -62659 (src/static_ic.cpp:119).  For
// any other seed the harness calls static_ic with ampt = 0 and then applies the perturbation
// itself with the reference's ran2() and the reference draw order (src/static_ic.cpp:114-159):
// z-rank, local k, y-rank, then the nry x npx plane x-fastest; each plane value is
// 1 + ampt*(ran2()-0.5) and multiplies TT.  Seed 62659 through this path equals the stock path
// bit for bit (checked by tests/test_oracle_ref.py).
//
// GPU mode (ref_run_gpu, ref_time_gpu): after the same set-up, every thread-rank runs the
// reference's own GPU time loop (src/main.cpp:234-275: gpu_alloc, gpu_upload, step_gpu,
// gpu_download) through its own copy of the reference GPU driver, _ref/libr3dgpu_r<rank>.so
// (see ref_gpu_entry.cpp); all ranks share the one device.
#include <dlfcn.h>
#include <omp.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <exception>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "communicate.hpp"
#include "fields.hpp"
#include "fluxes.hpp"
#include "grid.hpp"
#include "mpi.h"
#include "params.hpp"
#include "ran2.hpp"
#include "static_ic.hpp"
#include "step.hpp"
#include "topology.hpp"

namespace {

struct Job {
    std::vector<std::string> args;
    int nranks = 2;
    int seed = 62659;
    int nsteps = 0;
    int last_stages = 3;
    int omp_threads = 1;
    int fluxes_only = 0;  // after nsteps, run one FLUXES and return FU..FT in place of state
    int warmup = 0;       // untimed steps before the timed nsteps (timing runs)
    int gpu = 0;          // step with the reference GPU driver instead of src/step.cpp
    // outputs (global arrays, may be null)
    double* out3d = nullptr;   // 8 x NX*NY*NZ : ru rv rw ro tt bx by bz (or fu fv fw fr ft ...)
    double* out1d = nullptr;   // 14 x (NX | NY | NZ) packed: exx.. (NX) wyy.. (NY) zee.. (NZ) rkapa dkapa (NZ)
    double* scalars = nullptr; // dt timc timt timi umach tb nit
    double* seconds = nullptr; // wall time of the stepping loop (rank 0)
    std::string error;
};

void perturb_with_seed(const r3d::Params& p, const r3d::Derived& d, const r3d::Topology& t,
                       r3d::SimState& s, double ampt, int seed) {
    const int nx = d.nx, ny = d.ny, nz = d.nz;
    const int ilaph = p.ilap / 2;
    const int ixx = p.ix / 2, iyx = p.iy / 2;
    const int ip1 = ixx, ip2 = nx - ixx - 1, jp1 = iyx, jp2 = ny - iyx - 1;
    r3d::Ran2State st;
    st.idum = -seed;
    // Every rank replays the whole global draw sequence and keeps its own planes.
    for (int nnz = 1; nnz <= t.npez; ++nnz)
        for (int k = ilaph; k <= nz - 1 - ilaph; ++k)
            for (int nny = 1; nny <= t.npey; ++nny) {
                const int target = nny + t.npey * (nnz - 1) - 1;
                for (int jj = jp1; jj <= jp2; ++jj)
                    for (int ii = ip1; ii <= ip2; ++ii) {
                        double v = 1.0 + ampt * (r3d::ran2(st) - 0.5);
                        if (target == t.mype) s.ww1.at(ii, jj, k) = v;
                    }
            }
    for (int k = ilaph; k <= nz - 1 - ilaph; ++k)
        for (int j = jp1; j <= jp2; ++j)
            for (int i = ip1; i <= ip2; ++i) s.tt.at(i, j, k) *= s.ww1.at(i, j, k);
}

// Copy rank-local fields into the global arrays (interior + the global boundary ghosts).
void gather(const r3d::Params& p, const r3d::Derived& d, const r3d::Topology& t,
            const r3d::Field* const* f, int nf, double* out) {
    const long NX = p.npx + 2, NY = p.npy + 2, NZ = p.npz + 2;
    const long N = NX * NY * NZ;
    for (int kl = 0; kl < d.nz; ++kl) {
        bool kin = (kl >= 1 && kl <= d.nrz) || (kl == 0 && t.mypez == 0) ||
                   (kl == d.nz - 1 && t.mypez == t.npez - 1);
        if (!kin) continue;
        long kg = (long)t.mypez * d.nrz + kl;
        for (int jl = 0; jl < d.ny; ++jl) {
            bool jin = (jl >= 1 && jl <= d.nry) || (jl == 0 && t.mypey == 0) ||
                       (jl == d.ny - 1 && t.mypey == t.npey - 1);
            if (!jin) continue;
            long jg = (long)t.mypey * d.nry + jl;
            for (int q = 0; q < nf; ++q) {
                const double* src = f[q]->data() + (long)kl * d.nx * d.ny + (long)jl * d.nx;
                double* dst = out + q * N + kg * NX * NY + jg * NX;
                std::memcpy(dst, src, sizeof(double) * d.nx);
            }
        }
    }
}

void gather1d(const r3d::Params& p, const r3d::Derived& d, const r3d::Topology& t,
              const r3d::SimState& s, double* out) {
    const int NX = p.npx + 2, NY = p.npy + 2, NZ = p.npz + 2;
    const std::vector<double>* xs[4] = {&s.exx, &s.dxxdx, &s.d2xxdx2, &s.ddx};
    const std::vector<double>* ys[4] = {&s.wyy, &s.dyydy, &s.d2yydy2, &s.ddy};
    const std::vector<double>* zs[6] = {&s.zee, &s.dzzdz, &s.d2zzdz2, &s.ddz, &s.rkapa, &s.dkapa};
    if (t.mype == 0)
        for (int q = 0; q < 4; ++q) std::copy(xs[q]->begin(), xs[q]->end(), out + q * NX);
    double* yo = out + 4 * NX;
    if (t.mypez == 0)
        for (int jl = 0; jl < d.ny; ++jl) {
            bool jin = (jl >= 1 && jl <= d.nry) || (jl == 0 && t.mypey == 0) ||
                       (jl == d.ny - 1 && t.mypey == t.npey - 1);
            if (!jin) continue;
            int jg = t.mypey * d.nry + jl;
            for (int q = 0; q < 4; ++q) yo[q * NY + jg] = (*ys[q])[jl];
        }
    double* zo = yo + 4 * NY;
    if (t.mypey == 0)
        for (int kl = 0; kl < d.nz; ++kl) {
            bool kin = (kl >= 1 && kl <= d.nrz) || (kl == 0 && t.mypez == 0) ||
                       (kl == d.nz - 1 && t.mypez == t.npez - 1);
            if (!kin) continue;
            int kg = t.mypez * d.nrz + kl;
            for (int q = 0; q < 6; ++q) zo[q * NZ + kg] = (*zs[q])[kl];
        }
}

// One copy of the reference GPU driver (ref_gpu_entry.cpp), opened once per rank index and kept
// for the life of the process.
struct GpuCopy {
    void* (*alloc)(const r3d::Derived*) = nullptr;
    void (*upload)(void*, const r3d::SimState*) = nullptr;
    void (*download)(r3d::SimState*, void*) = nullptr;
    void (*step)(int, const r3d::Params*, const r3d::Derived*, const r3d::Topology*, void*, r3d::SimState*) = nullptr;
    void (*free_)(void*) = nullptr;
    int (*sync)(void) = nullptr;
};

constexpr int kMaxGpuCopies = 8;  // the copies oracle/Makefile builds

const GpuCopy& gpu_copy(int rank) {
    static std::mutex mu;
    static GpuCopy copies[kMaxGpuCopies];
    if (rank < 0 || rank >= kMaxGpuCopies) throw std::runtime_error("ref gpu: more ranks than driver copies");
    std::lock_guard<std::mutex> lk(mu);
    GpuCopy& c = copies[rank];
    if (c.alloc) return c;
    Dl_info info;
    if (!dladdr((void*)&gpu_copy, &info) || !info.dli_fname) throw std::runtime_error("ref gpu: dladdr failed");
    std::string dir(info.dli_fname);
    dir = dir.substr(0, dir.rfind('/') + 1);
    const std::string path = dir + "libr3dgpu_r" + std::to_string(rank) + ".so";
    void* h = dlopen(path.c_str(), RTLD_NOW | RTLD_LOCAL);
    if (!h) throw std::runtime_error(std::string("ref gpu: ") + dlerror());
    auto sym = [&](const char* name) {
        void* f = dlsym(h, name);
        if (!f) throw std::runtime_error(std::string("ref gpu: missing ") + name + " in " + path);
        return f;
    };
    GpuCopy n;
    n.alloc = (decltype(n.alloc))sym("r3dg_alloc");
    n.upload = (decltype(n.upload))sym("r3dg_upload");
    n.download = (decltype(n.download))sym("r3dg_download");
    n.step = (decltype(n.step))sym("r3dg_step");
    n.free_ = (decltype(n.free_))sym("r3dg_free");
    n.sync = (decltype(n.sync))sym("r3dg_sync");
    c = n;
    return c;
}

void rank_main(Job& job, int rank) {
    r3d_shim_bind_rank(rank);
    omp_set_num_threads(job.omp_threads);
    std::vector<char*> argv;
    static char prog[] = "3dmhd";
    argv.push_back(prog);
    std::vector<std::string> args = job.args;
    for (auto& a : args) argv.push_back(&a[0]);
    r3d::Params p;
    r3d::parse_args((int)argv.size(), argv.data(), p);
    int npe = 0;
    MPI_Comm_size(MPI_COMM_WORLD, &npe);
    r3d::Topology t = r3d::resolve_topology(npe, rank, p);
    r3d::Derived d = r3d::derive(p, npe, t.npey, t.npez);
    r3d::SimState s(d);
    // src/main.cpp:134-146
    r3d::build_grid_metrics(p, t, s);
    if (p.pzp == 0.0) {
        std::fill(s.rkapa.begin(), s.rkapa.end(), 1.0);
        std::fill(s.dkapa.begin(), s.dkapa.end(), 0.0);
    } else {
        for (int k = 0; k < d.nz; ++k) {
            double xe = s.zee[k];
            s.rkapa[k] = 1.0 + (d.rkapst - 1.0) / 2.0 * (1.0 + std::tanh((xe - p.pzp) / p.sigma));
            s.dkapa[k] = (d.rkapst - 1.0) / 2.0 / p.sigma / std::cosh((xe - p.pzp) / p.sigma) /
                         std::cosh((xe - p.pzp) / p.sigma);
        }
    }
    if (job.seed == 62659) {
        r3d::static_ic(MPI_COMM_WORLD, p, d, t, s);
    } else {
        r3d::Params p0 = p;
        double ampt = p.ampt;
        p0.ampt = 0.0;
        r3d::static_ic(MPI_COMM_WORLD, p0, d, t, s);
        if (ampt != 0.0) perturb_with_seed(p, d, t, s, ampt, job.seed);
    }
    s.timi = 0.0;
    r3d::communicate(MPI_COMM_WORLD, p, t, s);

    double wbuf[1] = {0.0}, wout[1];
    if (job.gpu) {
        // src/main.cpp:238-275; the rank's SimState is its own scalar mirror (step_gpu touches
        // only dt, nit, timc, timt, timi and tb of it)
        const GpuCopy& c = gpu_copy(rank);
        void* g = c.alloc(&d);
        c.upload(g, &s);
        for (int n = 1; n <= job.warmup; ++n) c.step(3, &p, &d, &t, g, &s);
        if (c.sync() != 0) throw std::runtime_error("ref gpu: device error before the timed steps");
        MPI_Allreduce(wbuf, wout, 1, MPI_DOUBLE, MPI_MIN, MPI_COMM_WORLD);
        auto t0 = std::chrono::steady_clock::now();
        for (int n = 1; n <= job.nsteps; ++n) c.step((n == job.nsteps) ? job.last_stages : 3, &p, &d, &t, g, &s);
        const int rc = c.sync();
        MPI_Allreduce(wbuf, wout, 1, MPI_DOUBLE, MPI_MIN, MPI_COMM_WORLD);
        auto t1 = std::chrono::steady_clock::now();
        if (rc != 0) throw std::runtime_error("ref gpu: device error in the timed steps");
        if (rank == 0 && job.seconds) *job.seconds = std::chrono::duration<double>(t1 - t0).count();
        if (job.out3d) c.download(&s, g);
        c.free_(g);
    } else {
        for (int n = 1; n <= job.warmup; ++n) r3d::step(3, MPI_COMM_WORLD, p, d, t, s);
        MPI_Allreduce(wbuf, wout, 1, MPI_DOUBLE, MPI_MIN, MPI_COMM_WORLD);
        auto t0 = std::chrono::steady_clock::now();
        for (int n = 1; n <= job.nsteps; ++n) {
            int ns = (n == job.nsteps) ? job.last_stages : 3;
            r3d::step(ns, MPI_COMM_WORLD, p, d, t, s);
        }
        MPI_Allreduce(wbuf, wout, 1, MPI_DOUBLE, MPI_MIN, MPI_COMM_WORLD);
        auto t1 = std::chrono::steady_clock::now();
        if (rank == 0 && job.seconds) *job.seconds = std::chrono::duration<double>(t1 - t0).count();
    }

    if (job.fluxes_only) {
        r3d::fluxes(p, d, t, s.rkapa.data(), s.dkapa.data(), s);
        const r3d::Field* f[8] = {&s.fu, &s.fv, &s.fw, &s.fr, &s.ft, &s.ro, &s.uu, &s.vv};
        if (job.out3d) gather(p, d, t, f, 8, job.out3d);
    } else {
        const r3d::Field* f[8] = {&s.ru, &s.rv, &s.rw, &s.ro, &s.tt, &s.bx, &s.by, &s.bz};
        if (job.out3d) gather(p, d, t, f, 8, job.out3d);
    }
    if (job.out1d) gather1d(p, d, t, s, job.out1d);
    if (rank == 0 && job.scalars) {
        job.scalars[0] = s.dt;
        job.scalars[1] = s.timc;
        job.scalars[2] = s.timt;
        job.scalars[3] = s.timi;
        job.scalars[4] = s.umach;
        job.scalars[5] = s.tb;
        job.scalars[6] = (double)s.nit;
    }
}

std::string g_last_error;

int run_job(Job& job) {
    const int nranks = job.nranks;
    r3d_shim_world_init(nranks);
    std::vector<std::thread> th;
    std::vector<std::string> errs(nranks);
    for (int r = 0; r < nranks; ++r)
        th.emplace_back([&, r] {
            try {
                rank_main(job, r);
            } catch (const std::exception& e) {
                errs[r] = e.what();
                try {
                    MPI_Abort(MPI_COMM_WORLD, 1);  // wakes ranks blocked in the shim
                } catch (...) {
                }
            } catch (...) {
            }
        });
    for (auto& x : th) x.join();
    g_last_error.clear();
    for (auto& e : errs)
        if (!e.empty()) g_last_error = e;
    return g_last_error.empty() ? 0 : 1;
}

}  // namespace

extern "C" {

// Run the reference CPU step.  args/nargs are reference CLI flags (src/params.cpp:113-224).
// Returns 0 on success, nonzero on failure (message via ref_last_error).
int ref_run(const char** args, int nargs, int nranks, int seed, int nsteps, int last_stages,
            int omp_threads, int fluxes_only, double* out3d, double* out1d, double* scalars,
            double* seconds) {
    Job job;
    for (int i = 0; i < nargs; ++i) job.args.emplace_back(args[i]);
    job.nranks = nranks;
    job.seed = seed;
    job.nsteps = nsteps;
    job.last_stages = last_stages;
    job.omp_threads = omp_threads;
    job.fluxes_only = fluxes_only;
    job.out3d = out3d;
    job.out1d = out1d;
    job.scalars = scalars;
    job.seconds = seconds;
    return run_job(job);
}

// Timing run: set-up, `warmup` untimed steps, then `nsteps` timed steps (wall time of the
// stepping loop on rank 0 into *seconds); only the scalars are returned (no gather).
int ref_time(const char** args, int nargs, int nranks, int seed, int warmup, int nsteps, int omp_threads,
             double* scalars, double* seconds) {
    Job job;
    for (int i = 0; i < nargs; ++i) job.args.emplace_back(args[i]);
    job.nranks = nranks;
    job.seed = seed;
    job.warmup = warmup;
    job.nsteps = nsteps;
    job.omp_threads = omp_threads;
    job.scalars = scalars;
    job.seconds = seconds;
    return run_job(job);
}

// The same two runs with the reference's own GPU driver (src/gpu.cpp) on every thread-rank:
// state after nsteps (ru rv rw ro tt bx by bz, downloaded as src/main.cpp:273 does) and timing.
int ref_run_gpu(const char** args, int nargs, int nranks, int seed, int nsteps, int last_stages,
                double* out3d, double* scalars, double* seconds) {
    Job job;
    for (int i = 0; i < nargs; ++i) job.args.emplace_back(args[i]);
    job.nranks = nranks;
    job.seed = seed;
    job.nsteps = nsteps;
    job.last_stages = last_stages;
    job.gpu = 1;
    job.out3d = out3d;
    job.scalars = scalars;
    job.seconds = seconds;
    return run_job(job);
}

int ref_time_gpu(const char** args, int nargs, int nranks, int seed, int warmup, int nsteps, double* scalars,
                 double* seconds) {
    Job job;
    for (int i = 0; i < nargs; ++i) job.args.emplace_back(args[i]);
    job.nranks = nranks;
    job.seed = seed;
    job.warmup = warmup;
    job.nsteps = nsteps;
    job.gpu = 1;
    job.scalars = scalars;
    job.seconds = seconds;
    return run_job(job);
}

const char* ref_last_error(void) { return g_last_error.c_str(); }

// RAN2 draws with the reference generator (src/ran2.cpp:13-32): n draws from idum=-seed.
void ref_ran2(int seed, int n, double* out) {
    r3d::Ran2State st;
    st.idum = -seed;
    for (int i = 0; i < n; ++i) out[i] = r3d::ran2(st);
}

}  // extern "C"
