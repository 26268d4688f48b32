// r3d_main.cpp - the command-line driver: the reference's main() with the GPU time loop
// (src/main.cpp:110-275) over the C ABI of include/r3d_gpu.h.
//
//     r3d_b200 [reference flags ...] [--backend gpu] [--dump-mode 0|1|2]
//
// Same flags, defaults and validation as the reference (r3d_params_parse), the same start-up
// line, progress line "NIT n  DT ..  TIMC ..  UMACH ..  WALL ..s (..s/step)" at the NSTEP0
// cadence and at the end, the same dt < 1e-8 underflow stop, and gstate dumps in the
// reference's binary format (src/main.cpp:42-93): gstate.start.000.0000 and
// gstate.step.000.NNNN.  The reference picks the dump policy at compile time (R3D_DUMP_MODE:
// 0 none, 1 start + final, 2 start + every NSTEP0 + final, default 2); here the same macro
// sets the default and --dump-mode overrides it.  There is one process and one GPU (the whole
// domain on the device), so the dump is the single rank 000 with the global extents.
//
// There is no CPU time loop: --backend cpu is refused (the reference CPU build is the CPU
// implementation); without --backend the GPU runs.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <string>
#include <vector>

#include "r3d_gpu.h"

#ifndef R3D_DUMP_MODE
#define R3D_DUMP_MODE 2
#endif

namespace {

[[noreturn]] void fatal(const std::string& msg) {
    std::fprintf(stderr, "%s\n", msg.c_str());
    std::fflush(stderr);
    std::exit(1);
}

void check(int rc, const char* what) {
    if (rc == R3D_OK) return;
    fatal(std::string("rast-3dmhd: ") + what + " failed (" + std::to_string(rc) + "): " + r3d_last_error());
}

double derived(const r3d_params& p, const char* name) {
    double v = 0.0;
    check(r3d_derived_get(&p, name, &v), name);
    return v;
}

struct HostState {
    int64_t nx = 0, ny = 0, nz = 0;
    std::vector<double> f[8];     // ru rv rw ro tt bx by bz
    std::vector<double> z[8];     // the RK accumulators zru .. ztt, zbx zby zbz (0 before a step)
    std::vector<double> line[14]; // exx dxxdx d2xxdx2 ddx wyy dyydy d2yydy2 ddy zee dzzdz d2zzdz2 ddz rkapa dkapa
    r3d_host_state view{};

    explicit HostState(const r3d_params& p) {
        r3d_dims(&p, &nx, &ny, &nz);
        const size_t n = (size_t)(nx * ny * nz);
        for (auto& a : f) a.assign(n, 0.0);
        for (auto& a : z) a.assign(n, 0.0);
        const int64_t len[14] = {nx, nx, nx, nx, ny, ny, ny, ny, nz, nz, nz, nz, nz, nz};
        for (int q = 0; q < 14; ++q) line[q].assign((size_t)len[q], 0.0);
        double** fp[8] = {&view.ru, &view.rv, &view.rw, &view.ro, &view.tt, &view.bx, &view.by, &view.bz};
        for (int q = 0; q < 8; ++q) *fp[q] = f[q].data();
        double** lp[14] = {&view.exx, &view.dxxdx, &view.d2xxdx2, &view.ddx, &view.wyy, &view.dyydy, &view.d2yydy2,
                           &view.ddy, &view.zee, &view.dzzdz, &view.d2zzdz2, &view.ddz, &view.rkapa, &view.dkapa};
        for (int q = 0; q < 14; ++q) *lp[q] = line[q].data();
    }
    double at(int q, int64_t i, int64_t j, int64_t k) const { return f[q][(size_t)((k * ny + j) * nx + i)]; }
};

// The start-up dt estimate of the log line (src/main.cpp:98-120): hydro limits only.
double initial_dt(const r3d_params& p, const HostState& s) {
    const double repr = derived(p, "repr"), cv = derived(p, "cv");
    double w[3] = {1e300, 1e300, 1e300};
    for (int64_t k = 1; k <= s.nz - 2; ++k)
        for (int64_t j = 1; j <= s.ny - 2; ++j)
            for (int64_t i = 1; i <= s.nx - 2; ++i) {
                const double ru = s.at(0, i, j, k), rv = s.at(1, i, j, k), rw = s.at(2, i, j, k);
                const double ro = s.at(3, i, j, k), tt = s.at(4, i, j, k);
                const double q = (ru * ru + rv * rv + rw * rw) * (1.0 / ro) * (1.0 / ro);
                const double uu = q + p.gamma * tt + 2.0 * std::sqrt(q * p.gamma * tt);
                const double dd = std::min(std::min(s.line[3][(size_t)i], s.line[7][(size_t)j]), s.line[11][(size_t)k]);
                w[0] = std::min(w[0], dd / std::sqrt(uu));
                w[1] = std::min(w[1], 0.5 * dd * dd * repr * cv * ro / s.line[12][(size_t)k]);
                w[2] = std::min(w[2], 0.375 * dd * dd * p.re * ro);
            }
    return p.sf * std::min(std::min(w[0], w[1]), w[2]);
}

// gstate dump, src/main.cpp:42-93: magic, counts, 13-int header, 27 scalars, 27 3D arrays and
// 14 1D arrays each preceded by its int64 length, int64 -1.  The RK accumulators zru..ztt and
// zbx..zbz are the device's (r3d_gpu_download_accumulators, interior cells).  `work` (after a
// step; null at the start) holds uu vv ww fu fv fw fr ft of the last step's third-stage input
// (r3d_gpu_download_work); the scratch arrays ww1..ww3, whose contents in the reference are
// whatever its last FLUXES sweep left, are written as zeros, and so is anything work lacks.
void write_gstate(const r3d_params& p, const HostState& s, const r3d_scalars& sc, const char* tag, int iter,
                  const std::vector<std::vector<double>>* work = nullptr) {
    char fname[256];
    std::snprintf(fname, sizeof fname, "gstate.%s.%03d.%04d", tag, 0, iter);
    FILE* fp = std::fopen(fname, "wb");
    if (!fp) fatal(std::string("rast-3dmhd: cannot open dump '") + fname + "'");
    auto w = [&](const void* v, size_t n) {
        if (std::fwrite(v, 1, n, fp) != n) fatal(std::string("rast-3dmhd: short write to '") + fname + "'");
    };
    const int32_t magic = 1129928788, nf = 27, n1 = 14;
    w(&magic, 4);
    w(&nf, 4);
    w(&n1, 4);
    const int32_t hdr[13] = {(int32_t)s.nx, (int32_t)s.ny, (int32_t)s.nz, 0, 0, 0, sc.nit, (int32_t)p.lmag,
                             (int32_t)p.ixcon, (int32_t)p.iycon, (int32_t)p.izcon, (int32_t)p.itcon, (int32_t)p.ibcon};
    w(hdr, sizeof hdr);
    const double scal[27] = {sc.dt,        sc.timc,          sc.timt,          sc.timi,          sc.umach,
                             p.re,         derived(p, "repr"), derived(p, "cv"), derived(p, "ocv"), derived(p, "ore"),
                             p.theta,      p.grav,           derived(p, "rkapst"), derived(p, "orm"), p.rm,
                             derived(p, "obeta"), derived(p, "omx"), derived(p, "omz"), p.sf,        p.ampt,
                             0.0,          derived(p, "hx"), derived(p, "h2x"), derived(p, "hy"), derived(p, "h2y"),
                             derived(p, "hz"), derived(p, "h2z")};
    w(scal, sizeof scal);
    // the reference's field order: ru rv rw ro tt uu vv ww fu fv fw fr ft zru zrv zrw zro ztt
    // ww1 ww2 ww3 bx by bz zbx zby zbz
    // (primaries 0-7, accumulators 8-15, work arrays 16-23, -1: not kept)
    const int order[27] = {0, 1, 2, 3, 4, 16, 17, 18, 19, 20, 21, 22, 23, 8,
                           9, 10, 11, 12, -1, -1, -1, 5, 6, 7, 13, 14, 15};
    const int64_t cnt = s.nx * s.ny * s.nz;
    std::vector<double> zeros((size_t)cnt, 0.0);
    for (int q = 0; q < 27; ++q) {
        w(&cnt, 8);
        const int o = order[q];
        const double* src = zeros.data();
        if (o >= 0 && o < 8) src = s.f[o].data();
        else if (o >= 8 && o < 16) src = s.z[o - 8].data();
        else if (o >= 16 && work && !(*work)[o - 16].empty()) src = (*work)[o - 16].data();
        w(src, (size_t)cnt * 8);
    }
    for (int q = 0; q < 14; ++q) {
        const int64_t c = (int64_t)s.line[q].size();
        w(&c, 8);
        w(s.line[q].data(), (size_t)c * 8);
    }
    const int64_t end = -1;
    w(&end, 8);
    std::fclose(fp);
}

// Restart (3dmhd.f:289-365, the Fortran driver's NSTART branch; the reference C++ aborts on it,
// src/main.cpp:150-152): dump number nstart of the NSTEP0-cadence dumps, i.e. the one written at
// NIT = nstart * nstep0, is read back from this driver's gstate file.  The fields - whole arrays,
// ghost planes included - replace the initial condition; NIT continues; as in the Fortran, the
// new run's time origin is TIMI = TIMI + TIMC of the dump with TIMC = 0, and TB is the dumped
// bottom plane's temperature.
void read_restart(const r3d_params& p, int nstart, HostState& s, r3d_scalars& sc) {
    char fname[256];
    std::snprintf(fname, sizeof fname, "gstate.step.%03d.%04d", 0, nstart * p.nstep0);
    FILE* fp = std::fopen(fname, "rb");
    if (!fp) fatal(std::string("rast-3dmhd: restart dump '") + fname + "' not found");
    auto rd = [&](void* v, size_t n) {
        if (std::fread(v, 1, n, fp) != n) fatal(std::string("rast-3dmhd: restart dump '") + fname + "' is truncated");
    };
    int32_t head[3], hdr[13];
    double scal[27];
    rd(head, sizeof head);
    if (head[0] != 1129928788 || head[1] != 27 || head[2] != 14)
        fatal(std::string("rast-3dmhd: '") + fname + "' is not a gstate dump");
    rd(hdr, sizeof hdr);
    rd(scal, sizeof scal);
    if (hdr[0] != s.nx || hdr[1] != s.ny || hdr[2] != s.nz || hdr[7] != p.lmag)
        fatal("rast-3dmhd: restart: grid size mismatch, no interpolation");
    // the reference's field order: ru rv rw ro tt uu vv ww fu fv fw fr ft zru .. ztt ww1 ww2 ww3 bx by bz ..
    const int field_of[27] = {0, 1, 2, 3, 4, -1, -1, -1, -1, -1, -1, -1, -1, -1,
                              -1, -1, -1, -1, -1, -1, -1, 5, 6, 7, -1, -1, -1};
    const int64_t cnt = s.nx * s.ny * s.nz;
    std::vector<double> skip((size_t)cnt);
    for (int q = 0; q < 27; ++q) {
        int64_t c = 0;
        rd(&c, 8);
        if (c != cnt) fatal("rast-3dmhd: restart: bad array length in the dump");
        const int f = field_of[q];
        rd(f >= 0 ? s.f[f].data() : skip.data(), (size_t)cnt * 8);
    }
    std::fclose(fp);
    sc.nit = hdr[6];
    sc.dt = scal[0];
    sc.timi = scal[3] + scal[1];  // TIMI = PAR1(64) + PAR1(65), 3dmhd.f:330
    sc.timc = 0.0;
    sc.timt = sc.timi;
    sc.umach = scal[4];
    sc.tb = s.f[4][(size_t)(((s.nz - 2) * s.ny + 1) * s.nx + 1)];  // TB = TT(2,2,NZ-ILAP/2), 3dmhd.f:358
}

}  // namespace

int main(int argc, char** argv) {
    int dump_mode = R3D_DUMP_MODE;
    std::vector<const char*> args;
    for (int a = 1; a < argc; ++a) {
        const std::string s = argv[a];
        if (s == "--dump-mode" && a + 1 < argc) {
            dump_mode = std::atoi(argv[++a]);
        } else if (s.rfind("--dump-mode=", 0) == 0) {
            dump_mode = std::atoi(s.c_str() + 12);
        } else {
            args.push_back(argv[a]);
        }
    }
    if (dump_mode < 0 || dump_mode > 2) fatal("rast-3dmhd: --dump-mode must be 0 (none), 1 (final) or 2 (periodic)");
    r3d_params p;
    check(r3d_params_default(&p), "r3d_params_default");
    bool backend_given = false;
    for (const char* a : args)
        if (std::strncmp(a, "--backend", 9) == 0) backend_given = true;
    check(r3d_params_parse((int)args.size(), args.data(), &p), "argument parsing");
    if (backend_given && p.backend != 1)
        fatal("rast-3dmhd: this binary runs the GPU time loop only (--backend gpu); the CPU backend is the "
              "reference build");
    p.backend = 1;
    const int nstart = p.nstart;  // a driver feature: the library sees a new start
    if (nstart < 0) fatal("rast-3dmhd: --nstart must be >= 0");
    p.nstart = 0;
    check(r3d_params_check(&p), "parameter check");

    HostState s(p);
    r3d_scalars sc{};
    check(r3d_setup_host(&p, &s.view, &sc), "initial condition");
    if (nstart > 0) read_restart(p, nstart, s, sc);
    const double dt0 = initial_dt(p, s);
    std::fprintf(stderr, "rast-3dmhd: NP=%d NPEY=%d NPEZ=%d  local %lldx%lldx%lld  NIT0=%d DT=%g NTOTAL=%d\n", 1, 1, 1,
                 (long long)s.nx, (long long)s.ny, (long long)s.nz, p.ntotal, dt0, p.ntotal);
    if (dump_mode != 0 && nstart == 0) write_gstate(p, s, sc, "start", 0);

    struct timespec wstart;
    clock_gettime(CLOCK_MONOTONIC, &wstart);
    auto wall_since = [&]() {
        struct timespec now;
        clock_gettime(CLOCK_MONOTONIC, &now);
        return (double)(now.tv_sec - wstart.tv_sec) + 1e-9 * (double)(now.tv_nsec - wstart.tv_nsec);
    };
    auto should_dump = [&](int nit, int nk) {
        if (dump_mode == 0) return false;
        if (dump_mode == 1) return nk == p.ntotal;
        return (nit % p.nstep0 == 0) || nk == p.ntotal;
    };
    auto should_log = [&](int nit, int nk) {
        if (dump_mode == 0) return (nit % p.nstep0 == 0) || nk == p.ntotal;
        return should_dump(nit, nk);
    };

    r3d_gpu* g = nullptr;
    check(r3d_gpu_create(&p, &g), "r3d_gpu_create");
    check(r3d_gpu_upload(g, &s.view, &sc), "r3d_gpu_upload");
    for (int nk = 1; nk <= p.ntotal; ++nk) {
        check(r3d_gpu_step(g, 3, &sc), "r3d_gpu_step");
        if (sc.dt < 1.0e-8) {
            std::fprintf(stderr, "rast-3dmhd: timestep underflow at NIT=%d\n", sc.nit);
            break;
        }
        if (should_log(sc.nit, nk)) {
            if (should_dump(sc.nit, nk)) {
                check(r3d_gpu_download(g, &s.view, nullptr), "r3d_gpu_download");
                double* zp[8];
                for (int q = 0; q < 8; ++q) zp[q] = s.z[q].data();
                check(r3d_gpu_download_accumulators(g, zp), "r3d_gpu_download_accumulators");
                // FP64: uu vv ww and, without density diffusion, fu..ft of the step's third stage
                std::vector<std::vector<double>> work(8);
                if (p.precision == R3D_PREC_FP64) {
                    double* wp[8] = {};
                    const size_t cnt = (size_t)(s.nx * s.ny * s.nz);
                    for (int q = 0; q < 8; ++q) {
                        if (q >= 3 && p.id != 0) continue;
                        work[q].assign(cnt, 0.0);
                        wp[q] = work[q].data();
                    }
                    check(r3d_gpu_download_work(g, wp), "r3d_gpu_download_work");
                }
                write_gstate(p, s, sc, "step", sc.nit, &work);
            }
            const double wall = wall_since();
            std::fprintf(stderr, "NIT %d  DT %g  TIMC %g  UMACH %g  WALL %.1fs (%.2fs/step)\n", sc.nit, sc.dt, sc.timc,
                         sc.umach, wall, wall / nk);
        }
    }
    check(r3d_gpu_download(g, &s.view, nullptr), "r3d_gpu_download");
    r3d_gpu_destroy(g);
    return 0;
}
