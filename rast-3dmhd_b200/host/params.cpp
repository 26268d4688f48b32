// params.cpp - configuration: defaults, the reference command line, derived constants.
//
// Defaults and flags follow include/params.hpp:26-113 and src/params.cpp:113-224 (same names,
// same "--key value" / "--key=value" forms, same boolean spellings, unknown flag = error).  The
// extensions --seed and --precision are added.  derive() reproduces src/params.cpp:29-64.
#include <cmath>
#include <cstddef>
#include <cstdlib>
#include <cstring>
#include <string>

#include "r3d_error.hpp"
#include "r3d_host.hpp"

namespace r3db {

namespace {
thread_local std::string t_error;

inline double widen(float x) { return (double)x; }

enum class Kind { Int, Dbl, Bool };
struct Flag {
    const char* name;
    Kind kind;
    size_t off;
};
#define I_(n, f) {n, Kind::Int, offsetof(r3d_params, f)}
#define D_(n, f) {n, Kind::Dbl, offsetof(r3d_params, f)}
#define B_(n, f) {n, Kind::Bool, offsetof(r3d_params, f)}
const Flag kFlags[] = {
    I_("--npx", npx), I_("--npy", npy), I_("--npz", npz), I_("--npey", npey), I_("--ix", ix),
    I_("--iy", iy), I_("--ilap", ilap), I_("--ngrid", ngrid), I_("--id", id), I_("--ncol", ncol),
    I_("--nrow", nrow), I_("--ixcon", ixcon), I_("--iycon", iycon), I_("--izcon", izcon),
    I_("--itcon", itcon), I_("--ibcon", ibcon), I_("--ncase", ncase), I_("--ncasep", ncasep),
    I_("--ntotal", ntotal), I_("--nstep0", nstep0), I_("--nstart", nstart), I_("--ntube", ntube),
    I_("--gpu", gpu_id), I_("--seed", seed),
    D_("--re", re), D_("--pr", pr), D_("--theta", theta), D_("--grav", grav), D_("--ry", r_y),
    D_("--ang", ang), D_("--rm", rm), D_("--beta", beta), D_("--pzp", pzp), D_("--sigma", sigma),
    D_("--polys", polys), D_("--tp", tp), D_("--tc", tc), D_("--xp", xp), D_("--yp", yp),
    D_("--zp", zp), D_("--xmax", xmax), D_("--ymax", ymax), D_("--zmax", zmax),
    D_("--ampt", ampt), D_("--ampb", ampb), D_("--bfh", bfh), D_("--bzp", bzp), D_("--qfh", qfh),
    D_("--gamma", gamma), D_("--hh", hh), D_("--dh", dh), D_("--dv", dv),
    D_("--tstart", tstart), D_("--toff", toff), D_("--rlax", rlax), D_("--xx1", xx1),
    D_("--xx2", xx2), D_("--yy1", yy1), D_("--yy2", yy2), D_("--zz1", zz1), D_("--zz2", zz2),
    D_("--xa", xa), D_("--xb", xb), D_("--xc", xc), D_("--xd", xd), D_("--ya", ya),
    D_("--yb", yb), D_("--yc", yc), D_("--yd", yd), D_("--za", za), D_("--zb", zb),
    D_("--zc", zc), D_("--zd", zd), D_("--xcent", xcent), D_("--zcent", zcent),
    D_("--rmax", rmax), D_("--cmt", cmt), D_("--a", a_tube), D_("--lambda", lambda),
    D_("--vz0", vz0), D_("--sff", sf),
    B_("--lrot", lrot), B_("--lmag", lmag), B_("--lpot", lpot), B_("--lrem", lrem),
    B_("--lshr", lshr),
};
#undef I_
#undef D_
#undef B_

bool truthy(const std::string& s) { return s == "1" || s == "true" || s == "yes" || s == "on"; }

}  // namespace

void set_error(const std::string& m) { t_error = m; }
void clear_error() { t_error.clear(); }

Derived derive(const r3d_params& p) {
    Derived d{};
    d.npx = p.npx;
    d.npy = p.npy;
    d.npz = p.npz;
    d.nx = (int64_t)p.npx + 2;
    d.ny = (int64_t)p.npy + 2;
    d.nz = (int64_t)p.npz + 2;
    d.c13 = widen(1.0f / 3.0f);
    d.c23 = 2.0 * d.c13;
    d.c43 = 4.0 * d.c13;
    d.gam[0] = widen(8.0f / 15.0f);
    d.gam[1] = widen(5.0f / 12.0f);
    d.gam[2] = widen(3.0f / 4.0f);
    d.zeta[0] = 0.0;
    d.zeta[1] = widen(-17.0f / 60.0f);
    d.zeta[2] = widen(-5.0f / 12.0f);
    d.hx = widen(0.5f * (float)(p.npx - 1));
    d.h2x = widen((float)(p.npx - 1) * (float)(p.npx - 1));
    d.hy = widen(0.5f * (float)(p.npy - 1));
    d.h2y = widen((float)(p.npy - 1) * (float)(p.npy - 1));
    d.hz = widen(0.5f * (float)(p.npz - 1));
    d.h2z = widen((float)(p.npz - 1) * (float)(p.npz - 1));
    d.repr = p.re * p.pr;
    d.ore = 1.0 / p.re;
    d.cv = 1.0 / (p.gamma - 1.0);
    d.ocv = 1.0 / d.cv;
    d.rkapst = (p.grav == 0.0) ? 1.0 : (p.polys + 1.0) * p.theta / p.grav;
    d.orm = p.lmag ? 1.0 / p.rm : 0.0;
    d.obeta = p.lmag ? 2.0 / p.beta : 0.0;
    d.omx = p.lrot ? std::sin(p.ang) / p.r_y : 0.0;
    d.omz = p.lrot ? std::cos(p.ang) / p.r_y : 0.0;
    return d;
}

void check_params(const r3d_params& p) {
    auto bad = [](const std::string& m) { throw std::invalid_argument(m); };
    if (p.ix != 2 || p.iy != 2 || p.ilap != 2)
        bad("stencil widths --ix/--iy/--ilap must be 2 (the stencil is radius 1)");
    if (p.npx < 3 || p.npy < 3 || p.npz < 5) bad("grid too small: need npx, npy >= 3 and npz >= 5");
    if (p.ixcon != 0 || p.iycon != 0)
        bad("non-periodic horizontal boundaries are not supported (the Fortran FLUXES stops on them too, "
            "3dmhdsub.f:1267-1280)");
    if (p.lshr) bad("LSHR is not supported (the reference aborts too)");
    if (p.lrem) bad("LREM is not supported (the reference aborts too)");
    if (p.rlax > 0.0) bad("flux relaxation (RLAX) is not supported (the reference aborts too)");
    if (p.id != 0) {
        // density diffusion, 3dmhdsub.f:1316-1386: its HORIZONTAL_MEAN exists for the uniform
        // grid only (3dmhdsub.f:3187-3190 stops otherwise)
        if (p.id != 1 && p.id != 2) bad("ID must be 0, 1 or 2");
        if (p.ngrid != 0) bad("ID (density diffusion) needs the uniform grid --ngrid 0, as the Fortran does");
        if (p.precision != R3D_PREC_FP64 || p.lmag)
            bad("ID (density diffusion) is available in the fp64 hydro form only");
    }
    if (!(p.itcon >= 0 && p.itcon <= 4)) bad("ITCON must be 0 .. 4 (others leave the top plane undefined)");
    if (p.itcon == 2 && p.precision != R3D_PREC_FP64)
        bad("ITCON 2 (embedded heat loss) is available in the fp64 form only");
    if (p.itcon == 3 && (p.precision != R3D_PREC_FP64 || p.lmag))
        bad("ITCON 3 (free top temperature) is available in the fp64 hydro form only");
    if (p.izcon != 0 && p.izcon != 1) bad("IZCON must be 0 or 1");
    if (p.nstart != 0)
        bad("restart (nstart != 0) is a driver feature: the r3d_b200 command line reads its own gstate "
            "dumps; the library starts from the state it is given");
    if (p.lmag && p.ntube != 0) bad("TUBE models are not supported (the reference aborts too)");
    if (p.ampb != 0.0 && !p.lmag) bad("AMPB magnetic layer requires LMAG");
    if (p.lmag && (p.rm == 0.0 || p.beta == 0.0)) bad("LMAG needs nonzero --rm and --beta");
    if (p.lmag && p.ibcon != 0) bad("IBCON must be 0 (Bz = 0 at top and bottom)");
    if (p.precision != R3D_PREC_FP64 && p.precision != R3D_PREC_FP32BULK)
        bad("--precision must be fp64 or fp32bulk");
    if (p.precision == R3D_PREC_FP32BULK && p.lmag)
        bad("the fp32bulk form covers hydro (lmag = 0) only");
    if (p.ngrid < 0 || p.ngrid > 2) bad("NGRID must be 0, 1 or 2");
    if (p.seed <= 0) bad("--seed must be positive");
}

}  // namespace r3db

using namespace r3db;

extern "C" {

const char* r3d_last_error(void) { return t_error.c_str(); }

int r3d_params_default(r3d_params* p) {
    if (!p) return R3D_EINVAL;
    std::memset(p, 0, sizeof(*p));
    p->npx = 504;
    p->npy = 504;
    p->npz = 2048;
    p->npey = 8;
    p->ix = p->iy = p->ilap = 2;
    p->ngrid = 1;
    p->itcon = 1;
    p->ncase = p->ncasep = 1;
    p->ntotal = 1000;
    p->nstep0 = 100;
    p->re = 2.0;
    p->pr = widen(5.0e-2f);
    p->theta = 2.5e-1;
    p->grav = 6.25e-1;
    p->tp = 2.0;
    p->xp = 10.0;
    p->yp = 10.0;
    p->xmax = 20.0;
    p->ymax = 20.0;
    p->zmax = 40.0;
    p->ampt = widen(5.0e-3f);
    p->gamma = widen(5.0f / 3.0f);
    p->hh = 1.0;
    p->xx1 = -7.0;
    p->xx2 = 7.0;
    p->yy1 = -7.0;
    p->yy2 = 7.0;
    p->zz1 = -2.0;
    p->zz2 = 1.0e-2;
    p->xa = 0.5;
    p->xb = 0.48;
    p->xc = 28.0;
    p->xd = 0.025;
    p->ya = 0.5;
    p->yb = 0.48;
    p->yc = 28.0;
    p->yd = 0.025;
    p->za = 0.65;
    p->zb = 1.0;
    p->zc = 5.0;
    p->zd = 0.2;
    p->sf = widen(0.315f);
    p->seed = 62659;
    p->precision = R3D_PREC_FP64;
    return R3D_OK;
}

int r3d_params_parse(int argc, const char* const* argv, r3d_params* p) {
    return guarded([&] {
        if (!p || (argc > 0 && !argv)) throw std::invalid_argument("null argument");
        for (int a = 0; a < argc; ++a) {
            std::string arg = argv[a];
            auto value_of = [&](const std::string& name) -> std::string {
                if (arg.size() > name.size() && arg[name.size()] == '=')
                    return arg.substr(name.size() + 1);
                if (a + 1 >= argc) throw std::invalid_argument("missing value for " + name);
                return argv[++a];
            };
            auto is = [&](const std::string& name) {
                return arg == name || (arg.rfind(name, 0) == 0 && arg.size() > name.size() &&
                                       arg[name.size()] == '=');
            };
            if (is("--backend")) {
                std::string v = value_of("--backend");
                if (v == "cpu") p->backend = 0;
                else if (v == "gpu") p->backend = 1;
                else throw std::invalid_argument("--backend must be 'cpu' or 'gpu'");
                continue;
            }
            if (is("--precision")) {
                std::string v = value_of("--precision");
                if (v == "fp64") p->precision = R3D_PREC_FP64;
                else if (v == "fp32bulk") p->precision = R3D_PREC_FP32BULK;
                else throw std::invalid_argument("--precision must be 'fp64' or 'fp32bulk'");
                continue;
            }
            bool done = false;
            for (const Flag& f : kFlags) {
                if (!is(f.name)) continue;
                std::string v = value_of(f.name);
                char* base = (char*)p + f.off;
                if (f.kind == Kind::Int) *(int*)base = std::atoi(v.c_str());
                else if (f.kind == Kind::Dbl) *(double*)base = std::atof(v.c_str());
                else *(int*)base = truthy(v) ? 1 : 0;
                done = true;
                break;
            }
            if (!done) throw std::invalid_argument("unknown option '" + arg + "'");
        }
    });
}

int r3d_params_check(const r3d_params* p) {
    return guarded([&] {
        if (!p) throw std::invalid_argument("null params");
        check_params(*p);
    });
}

int r3d_derived_get(const r3d_params* p, const char* name, double* out) {
    return guarded([&] {
        if (!p || !name || !out) throw std::invalid_argument("null argument");
        Derived d = derive(*p);
        struct {
            const char* n;
            double v;
        } tab[] = {{"c13", d.c13},     {"c23", d.c23},     {"c43", d.c43},       {"gam1", d.gam[0]},
                   {"gam2", d.gam[1]}, {"gam3", d.gam[2]}, {"zeta1", d.zeta[1]}, {"zeta2", d.zeta[2]},
                   {"hx", d.hx},       {"h2x", d.h2x},     {"hy", d.hy},         {"h2y", d.h2y},
                   {"hz", d.hz},       {"h2z", d.h2z},     {"repr", d.repr},     {"ore", d.ore},
                   {"cv", d.cv},       {"ocv", d.ocv},     {"rkapst", d.rkapst}, {"orm", d.orm},
                   {"obeta", d.obeta}, {"omx", d.omx},     {"omz", d.omz}};
        for (auto& e : tab)
            if (std::strcmp(e.n, name) == 0) {
                *out = e.v;
                return;
            }
        throw std::invalid_argument(std::string("unknown derived constant ") + name);
    });
}

int r3d_dims(const r3d_params* p, int64_t* nx, int64_t* ny, int64_t* nz) {
    if (!p) return R3D_EINVAL;
    if (nx) *nx = (int64_t)p->npx + 2;
    if (ny) *ny = (int64_t)p->npy + 2;
    if (nz) *nz = (int64_t)p->npz + 2;
    return R3D_OK;
}

const char* r3d_version(void) { return "rast3d-b200 0.1 (sm_100a)"; }

}  // extern "C"
