// setup.cpp - one-time host set-up: grid metrics, conductivity, static polytrope, RAN2
// perturbation, periodic ghosts.
//
// The reference computes these per MPI rank (src/grid.cpp, src/static_ic.cpp) and the rank
// blocks stitch into one global domain; this file builds the stitched global result directly:
//  * y/z metrics: ghost 0 -> coordinate 0, interior g -> the (g-1)-th uniform computational
//    point, ghost np+1 -> coordinate 1 (src/grid.cpp:169-276 as assembled over ranks; the
//    per-rank code reads past its table when a direction has a single rank, so the global
//    result is the multi-rank one).
//  * RAN2 draw order: the reference draws plane by plane in (z-rank, local k, y-rank, rows,
//    x fastest) order (src/static_ic.cpp:122-153); because ranks own contiguous z and y
//    ranges this is the global (k, j, i) order for every decomposition.
// Arithmetic (association, single-precision seeds, libm calls) matches the reference.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <vector>

#include "r3d_error.hpp"
#include "r3d_host.hpp"

namespace r3db {

namespace {
inline double widen(float x) { return (double)x; }
}  // namespace

// ---- MKGRID (src/grid.cpp:28-146) --------------------------------------------------------
void map_coordinate(const r3d_params& p, double sc, int axis, double& sphys, double& dsds,
                    double& d2sds2) {
    const double pi = 2.0 * std::asin(1.0);
    const double smax = axis == 1 ? p.xmax : (axis == 2 ? p.ymax : p.zmax);
    if (p.ngrid == 0) {
        sphys = sc * smax;
        dsds = 1.0 / smax;
        d2sds2 = 0.0;
        return;
    }
    if (p.ngrid == 1) {
        const double s1 = axis == 1 ? p.xx1 : (axis == 2 ? p.yy1 : p.zz1);
        const double s2 = axis == 1 ? p.xx2 : (axis == 2 ? p.yy2 : p.zz2);
        const double a1 = (s2 - s1) / smax;
        const double a3 = std::atan(s1);
        const double a2 = std::atan(s2) - a3;
        if (sc == 0.0)
            sphys = 0.0;
        else if (sc == 1.0)
            sphys = smax;
        else
            sphys = (std::tan(a2 * sc + a3) - s1) / a1;
        dsds = a1 / a2 / (1.0 + (s1 + a1 * sphys) * (s1 + a1 * sphys));
        const double t = (s1 + a1 * sphys);
        const double den = (1.0 + t * t);
        d2sds2 = -2.0 * a1 * a1 * t / a2 / (den * den);
        return;
    }
    // ngrid == 2: two-arctan stretch
    const double a = axis == 1 ? p.xa : (axis == 2 ? p.ya : p.za);
    const double b = axis == 1 ? p.xb : (axis == 2 ? p.yb : p.zb);
    const double c = axis == 1 ? p.xc : (axis == 2 ? p.yc : p.zc);
    const double dp = axis == 1 ? p.xd : (axis == 2 ? p.yd : p.zd);
    if (c <= 1.0e-9) {
        sphys = sc * smax;
        dsds = 1.0 / smax;
        d2sds2 = 0.0;
        return;
    }
    using std::atan;
    using std::log;
    const double sh = (1.0 - dp) * pi /
                      (dp * atan((a - b) * c) + 2.0 * atan(b * c) - dp * atan((a + b) * c));
    const double sk =
        2.0 * c * pi * smax /
        (2.0 * c * pi +
         sh * (2.0 * c *
                   (atan((a - b) * c) * (a - b) - atan((a + b) * c) * (a + b) +
                    atan((a - b - 1.0) * c) + atan((a + b - 1.0) * c) * (a + b - 1.0) +
                    atan((1.0 - a + b) * c) * (a - b)) -
               log(1.0 + (a - b) * (a - b) * c * c) + log(1.0 + (a + b) * (a + b) * c * c) -
               log(1.0 + (a + b - 1.0) * (a + b - 1.0) * c * c) +
               log(1.0 + (1.0 - a + b) * (1.0 - a + b) * c * c)));
    dsds = 1.0 / (sk * (1.0 + sh / pi * (atan(c * (sc - a - b)) + atan(c * (a - sc - b)))));
    d2sds2 = -dsds * dsds * dsds * c * sh * sk / pi *
             (1.0 / (1.0 + c * c * (a + b - sc) * (a + b - sc)) -
              1.0 / (1.0 + c * c * (a - b - sc) * (a - b - sc)));
    sphys = sk / (2.0 * c * pi) *
            (2.0 * c * pi * sc +
             sh * (2.0 * c *
                       (atan((a - b) * c) * (a - b) - atan((a + b) * c) * (a + b) +
                        atan((a - b - sc) * c) * sc + atan((a + b - sc) * c) * (a + b - sc) +
                        atan((sc - a + b) * c) * (a - b)) -
                   log(1.0 + (a - b) * (a - b) * c * c) + log(1.0 + (a + b) * (a + b) * c * c) -
                   log(1.0 + (a + b - sc) * (a + b - sc) * c * c) +
                   log(1.0 + (sc - a + b) * (sc - a + b) * c * c)));
    if (sc == 0.0) sphys = 0.0;
    if (sc == 1.0) sphys = smax;
}

Metrics build_metrics(const r3d_params& p, const Derived& d) {
    Metrics m;
    // x (src/grid.cpp:148-167): points 1..npx carry the metric; the two ghosts stay 0.
    {
        Line& L = m.x;
        const int64_t n = d.nx;
        L.s.assign(n, 0.0);
        L.d1.assign(n, 0.0);
        L.d2.assign(n, 0.0);
        L.dd.assign(n, 0.0);
        const double orx = widen(1.0f / (float)(p.npx - 1));
        std::vector<double> sc(n, 0.0);
        for (int i = 0; i < p.npx - 1; ++i) sc[i + 1] = i * orx;
        sc[1] = 0.0;
        sc[p.npx] = 1.0;
        for (int i = 1; i <= p.npx; ++i) {
            map_coordinate(p, sc[i], 1, L.s[i], L.d1[i], L.d2[i]);
            L.dd[i] = orx * (1.0 / L.d1[i]);
        }
    }
    // y and z, stitched over ranks.
    for (int axis = 2; axis <= 3; ++axis) {
        Line& L = axis == 2 ? m.y : m.z;
        const int np = axis == 2 ? p.npy : p.npz;
        const int64_t n = (int64_t)np + 2;
        L.s.assign(n, 0.0);
        L.d1.assign(n, 0.0);
        L.d2.assign(n, 0.0);
        L.dd.assign(n, 0.0);
        const double o = widen(1.0f / (float)(np - 1));
        for (int64_t g = 0; g < n; ++g) {
            double sc;
            if (g <= 1)
                sc = 0.0;  // ghost and first point both sit at computational 0
            else if (g >= np)
                sc = 1.0;  // last point and ghost both sit at computational 1
            else
                sc = (double)(g - 1) * o;
            map_coordinate(p, sc, axis, L.s[g], L.d1[g], L.d2[g]);
        }
        for (int64_t g = 0; g < n; ++g) L.dd[g] = o * (1.0 / L.d1[g]);
    }
    // conductivity (src/main.cpp:135-146)
    m.rkapa.assign(d.nz, 1.0);
    m.dkapa.assign(d.nz, 0.0);
    if (p.pzp != 0.0) {
        for (int64_t k = 0; k < d.nz; ++k) {
            const double xe = m.z.s[k];
            m.rkapa[k] = 1.0 + (d.rkapst - 1.0) / 2.0 * (1.0 + std::tanh((xe - p.pzp) / p.sigma));
            m.dkapa[k] = (d.rkapst - 1.0) / 2.0 / p.sigma / std::cosh((xe - p.pzp) / p.sigma) /
                         std::cosh((xe - p.pzp) / p.sigma);
        }
    }
    return m;
}

// ---- RAN2 (src/ran2.cpp:13-32) ----------------------------------------------------------
double Ran2::next() {
    constexpr int M = 714025, IA = 1366, IC = 150889;
    const double rm = widen(1.0f / 714025.0f);
    if (idum_ < 0) {
        idum_ = (IC - idum_) % M;
        for (int j = 0; j < 97; ++j) {
            idum_ = (IA * idum_ + IC) % M;
            table_[j] = idum_;
        }
        idum_ = (IA * idum_ + IC) % M;
        iy_ = idum_;
    }
    const int j = 1 + (97 * iy_) / M;
    if (j < 1 || j > 97) throw Error(R3D_EINVAL, "RAN2 table index out of range");
    iy_ = table_[j - 1];
    const double r = (double)iy_ * rm;
    idum_ = (IA * idum_ + IC) % M;
    table_[j - 1] = idum_;
    return r;
}

// ---- static polytrope (src/ode.cpp:20-174: DERIVS + Bulirsch-Stoer with rational
//      extrapolation, fixed step 1/(npz-1), eps 1e-12) ------------------------------------
namespace {
constexpr int kMaxVar = 2, kStages = 11, kUsed = 7;
constexpr int kSeq[kStages] = {2, 4, 6, 8, 12, 16, 24, 32, 48, 64, 96};

struct Profile {
    const r3d_params& p;
    double rkapst;

    void rhs(double zz, const double* y, double* f) const {
        double z, dzdz, unused;
        map_coordinate(p, zz, 3, z, dzdz, unused);
        const double kap =
            (p.pzp == 0.0) ? 1.0 : 1.0 + (rkapst - 1.0) / 2.0 * (1.0 + std::tanh((z - p.pzp) / p.sigma));
        f[0] = p.theta / kap / dzdz;
        f[1] = p.grav / (1.0 + y[0]) / dzdz;
    }

    // modified midpoint over htot in nstp substeps
    void midpoint(const double* y, const double* f0, double x0, double htot, int nstp,
                  double* out) const {
        const double h = htot / nstp;
        double a[kMaxVar], b[kMaxVar], f[kMaxVar];
        for (int i = 0; i < kMaxVar; ++i) {
            a[i] = y[i];
            b[i] = y[i] + h * f0[i];
        }
        double x = x0 + h;
        rhs(x, b, f);
        const double h2 = 2.0 * h;
        for (int n = 1; n < nstp; ++n) {
            for (int i = 0; i < kMaxVar; ++i) {
                const double t = a[i] + h2 * f[i];
                a[i] = b[i];
                b[i] = t;
            }
            x += h;
            rhs(x, b, f);
        }
        for (int i = 0; i < kMaxVar; ++i) out[i] = 0.5 * (a[i] + b[i] + h * f[i]);
    }

    // diagonal rational extrapolation (tableau t, abscissae xs)
    static void extrapolate(int iest, double xest, const double* yest, double* yz,
                            double t[kMaxVar][kUsed], double* dy, double* xs) {
        xs[iest - 1] = xest;
        if (iest == 1) {
            for (int j = 0; j < kMaxVar; ++j) {
                yz[j] = yest[j];
                t[j][0] = yest[j];
                dy[j] = yest[j];
            }
            return;
        }
        const int m1 = iest < kUsed ? iest : kUsed;
        double fx[kUsed + 1];
        for (int k = 0; k < m1 - 1; ++k) fx[k + 1] = xs[iest - k - 2] / xest;
        for (int j = 0; j < kMaxVar; ++j) {
            double yy = yest[j], v = t[j][0], c = yy, ddy = 0.0;
            t[j][0] = yy;
            for (int k = 1; k < m1; ++k) {
                const double b1 = fx[k] * v;
                double b = b1 - c;
                if (b != 0.0) {
                    b = (c - v) / b;
                    ddy = c * b;
                    c = b1 * b;
                } else {
                    ddy = v;
                }
                v = t[j][k];
                t[j][k] = ddy;
                yy += ddy;
            }
            dy[j] = ddy;
            yz[j] = yy;
        }
    }

    // one Bulirsch-Stoer step; returns the step taken
    double bs_step(double* y, const double* f, double& x, double htry) const {
        double h = htry;
        const double x0 = x;
        double y0[kMaxVar], f0[kMaxVar], yseq[kMaxVar], yerr[kMaxVar], t[kMaxVar][kUsed],
            xs[kStages];
        for (int i = 0; i < kMaxVar; ++i) {
            y0[i] = y[i];
            f0[i] = f[i];
        }
        for (;;) {
            for (int i = 1; i <= kStages; ++i) {
                midpoint(y0, f0, x0, h, kSeq[i - 1], yseq);
                const double xest = (h / kSeq[i - 1]) * (h / kSeq[i - 1]);
                extrapolate(i, xest, yseq, y, t, yerr, xs);
                double emax = 0.0;
                for (int j = 0; j < kMaxVar; ++j) {
                    const double e = std::fabs(yerr[j] / y[j]);
                    if (e > emax) emax = e;
                }
                emax /= 1.0e-12;
                if (emax < 1.0) {
                    x += h;
                    return h;
                }
            }
            h = 0.25 * h / std::pow(2.0, double((kStages - kUsed) / 2));
            if (x + h == x) throw Error(R3D_ENUMERIC, "static profile: step size underflow");
        }
    }
};
}  // namespace

void static_profile(const r3d_params& p, std::vector<double>& T, std::vector<double>& R) {
    const int npz = p.npz;
    T.assign(npz, 0.0);
    R.assign(npz, 0.0);
    Profile prof{p, (p.grav == 0.0) ? 1.0 : (p.polys + 1.0) * p.theta / p.grav};
    const double h = widen(1.0f / (float)(npz - 1));
    double y[2] = {0.0, 0.0}, zz = 0.0;
    T[0] = 1.0;
    R[0] = 1.0;
    for (int k = 1; k < npz; ++k) {
        double f[2];
        prof.rhs(zz, y, f);
        const double did = prof.bs_step(y, f, zz, h);
        if (did != h) throw Error(R3D_ENUMERIC, "static profile: step was reduced");
        T[k] = 1.0 + y[0];
        R[k] = std::exp(y[1]) / (1.0 + y[0]);
    }
}

void fill_ghosts(double* f, int64_t nx, int64_t ny, int64_t nz) {
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < nz; ++k) {
        double* pl = f + k * nx * ny;
        std::memcpy(pl, pl + (ny - 2) * nx, sizeof(double) * nx);
        std::memcpy(pl + (ny - 1) * nx, pl + nx, sizeof(double) * nx);
        for (int64_t j = 0; j < ny; ++j) {
            pl[j * nx] = pl[j * nx + nx - 2];
            pl[j * nx + nx - 1] = pl[j * nx + 1];
        }
    }
}

IcColumns ic_columns(const r3d_params& p, int z0, int nz) {
    if (z0 < 0 || nz < 1 || z0 + nz > p.npz) throw std::invalid_argument("z range outside the domain");
    const Derived d = derive(p);
    const int64_t NZ = (int64_t)nz + 2, NZG = d.nz;
    IcColumns c;
    std::vector<double> T, R;
    static_profile(p, T, R);
    c.tb = T[p.npz - 1];
    c.rb = R[p.npz - 1];
    c.t.assign(NZ, 0.0);
    c.r.assign(NZ, 0.0);
    c.bfac.assign(NZ, 0.0);
    // src/static_ic.cpp:53-89 stitched over the ranks: ghost top = T(0), interior k = T(k-1),
    // ghost bottom = tb
    for (int64_t k = 0; k < NZ; ++k) {
        const int64_t kg = z0 + k;
        c.t[k] = kg == 0 ? T[0] : (kg == NZG - 1 ? c.tb : T[kg - 1]);
        c.r[k] = kg == 0 ? R[0] : (kg == NZG - 1 ? c.rb : R[kg - 1]);
    }
    if (p.lmag) {
        // magnetic layer (src/static_ic.cpp:94-108)
        const Metrics m = build_metrics(p, d);
        const double cln = widen(-4.0f * logf(2.0f)) / (p.bfh * p.bfh);
        for (int64_t k = 0; k < NZ; ++k) {
            const int64_t kg = z0 + k;
            if (kg < 1 || kg > NZG - 2) continue;
            const double z = m.z.s[kg];
            c.bfac[k] = p.ampb * std::exp(cln * (z - p.bzp) * (z - p.bzp));
        }
    }
    return c;
}

void setup_lines(const r3d_params& p, const r3d_host_state& st, int z0, int nz) {
    const Derived d = derive(p);
    const int64_t NZ = (int64_t)nz + 2;
    const Metrics m = build_metrics(p, d);
    auto put = [](double* dst, const std::vector<double>& v) {
        if (dst) std::memcpy(dst, v.data(), sizeof(double) * v.size());
    };
    put(st.exx, m.x.s); put(st.dxxdx, m.x.d1); put(st.d2xxdx2, m.x.d2); put(st.ddx, m.x.dd);
    put(st.wyy, m.y.s); put(st.dyydy, m.y.d1); put(st.d2yydy2, m.y.d2); put(st.ddy, m.y.dd);
    auto putz = [&](double* dst, const std::vector<double>& v) {
        if (dst) std::memcpy(dst, v.data() + z0, sizeof(double) * (size_t)NZ);
    };
    putz(st.zee, m.z.s); putz(st.dzzdz, m.z.d1); putz(st.d2zzdz2, m.z.d2); putz(st.ddz, m.z.dd);
    putz(st.rkapa, m.rkapa); putz(st.dkapa, m.dkapa);
}

// temperature perturbation draws (src/static_ic.cpp:114-159): global (k, j, i) order over the
// interior planes 1 .. npz; a slab skips the draws of the interior planes above it
PerturbationDraws::PerturbationDraws(const r3d_params& p, int z0, int nz)
    : rng_(-p.seed), per_plane_((int64_t)p.npx * p.npy) {
    const int64_t NZG = (int64_t)p.npz + 2, NZ = (int64_t)nz + 2;
    const int64_t kfirst = std::max<int64_t>(1, z0), klast = std::min<int64_t>(NZG - 2, z0 + NZ - 1);
    first_ = kfirst - z0;
    last_ = p.ampt != 0.0 ? klast - z0 : first_ - 1;
    if (p.ampt != 0.0)
        for (int64_t n = 0; n < (kfirst - 1) * per_plane_; ++n) rng_.next();
}

void PerturbationDraws::next_plane(double* out) {
    for (int64_t n = 0; n < per_plane_; ++n) out[n] = rng_.next();
}

// The initial state on global planes z0 .. z0+nz+1 (the whole domain: z0 = 0, nz = npz); the z
// metric lines are written from global index z0 on, nz+2 entries.
void setup_state(const r3d_params& p, const r3d_host_state& st, r3d_scalars& sc, int z0, int nz) {
    check_params(p);
    if (z0 < 0 || nz < 1 || z0 + nz > p.npz) throw std::invalid_argument("z range outside the domain");
    const Derived d = derive(p);
    const int64_t NX = d.nx, NY = d.ny, NZ = (int64_t)nz + 2;
    auto need = [](const double* a, const char* n) {
        if (!a) throw std::invalid_argument(std::string("r3d_host_state.") + n + " is NULL");
    };
    need(st.ru, "ru"); need(st.rv, "rv"); need(st.rw, "rw"); need(st.ro, "ro"); need(st.tt, "tt");
    if (p.lmag) { need(st.bx, "bx"); need(st.by, "by"); need(st.bz, "bz"); }
    setup_lines(p, st, z0, nz);

    // zero every field plane by plane over the host threads (the first touch of fresh pages
    // is most of the set-up time on large grids)
    for (double* a : {st.ru, st.rv, st.rw, st.ro, st.tt, st.bx, st.by, st.bz}) {
        if (!a || ((a == st.bx || a == st.by || a == st.bz) && !p.lmag)) continue;
#pragma omp parallel for schedule(static)
        for (int64_t k = 0; k < NZ; ++k) std::memset(a + k * NX * NY, 0, sizeof(double) * NX * NY);
    }

    const IcColumns c = ic_columns(p, z0, nz);
    auto at = [&](int64_t i, int64_t j, int64_t k) { return i + NX * (j + NY * k); };
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < NZ; ++k)
        for (int64_t j = 1; j <= NY - 2; ++j)
            for (int64_t i = 1; i <= NX - 2; ++i) {
                st.tt[at(i, j, k)] = c.t[k];
                st.ro[at(i, j, k)] = c.r[k];
            }
    if (p.lmag) {
        // magnetic layer (src/static_ic.cpp:94-108): Bx over whole interior planes, and the
        // density correction with the unperturbed T
#pragma omp parallel for schedule(static)
        for (int64_t k = 0; k < NZ; ++k) {
            const int64_t kg = z0 + k;
            if (kg < 1 || kg > d.nz - 2) continue;
            for (int64_t n = at(0, 0, k); n < at(0, 0, k + 1); ++n) st.bx[n] = c.bfac[k];
            for (int64_t j = 1; j <= NY - 2; ++j)
                for (int64_t i = 1; i <= NX - 2; ++i) {
                    const int64_t n = at(i, j, k);
                    st.ro[n] = st.ro[n] - st.bx[n] * st.bx[n] / st.tt[n] * d.obeta;
                }
        }
    }
    PerturbationDraws draws(p, z0, nz);
    std::vector<double> plane((size_t)p.npx * p.npy);
    for (int64_t k = draws.first(); k <= draws.last(); ++k) {
        draws.next_plane(plane.data());
        const double* u = plane.data();
        for (int64_t j = 1; j <= NY - 2; ++j)
            for (int64_t i = 1; i <= NX - 2; ++i) {
                const double w = 1.0 + p.ampt * (*u++ - 0.5);
                st.tt[at(i, j, k)] *= w;
            }
    }
    for (double* a : {st.ru, st.rv, st.rw, st.tt, st.ro}) fill_ghosts(a, NX, NY, NZ);
    if (p.lmag)
        for (double* a : {st.bx, st.by, st.bz}) fill_ghosts(a, NX, NY, NZ);
    sc.dt = 0.0;
    sc.timc = 0.0;
    sc.timt = 0.0;
    sc.timi = 0.0;
    sc.umach = 0.0;
    sc.tb = c.tb;
    sc.nit = 0;
}

}  // namespace r3db

using namespace r3db;

extern "C" {

int r3d_setup_host(const r3d_params* p, r3d_host_state* st, r3d_scalars* sc) {
    return guarded([&] {
        if (!p || !st || !sc) throw std::invalid_argument("null argument");
        setup_state(*p, *st, *sc, 0, p->npz);
    });
}

int r3d_setup_host_slab(const r3d_params* p, int z0, int nz, r3d_host_state* st, r3d_scalars* sc) {
    return guarded([&] {
        if (!p || !st || !sc) throw std::invalid_argument("null argument");
        setup_state(*p, *st, *sc, z0, nz);
    });
}

int r3d_static_profile(const r3d_params* p, double* t, double* r) {
    return guarded([&] {
        if (!p || !t || !r) throw std::invalid_argument("null argument");
        std::vector<double> T, R;
        static_profile(*p, T, R);
        std::memcpy(t, T.data(), sizeof(double) * T.size());
        std::memcpy(r, R.data(), sizeof(double) * R.size());
    });
}

}  // extern "C"
