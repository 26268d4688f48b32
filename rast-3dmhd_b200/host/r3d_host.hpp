// r3d_host.hpp - host-side model of the run: configuration, derived constants, grid metrics
// and the initial condition on the single global domain.
//
// Everything here runs once per run on the CPU.  The floating-point expressions reproduce the
// reference's (src/params.cpp:14-66, src/grid.cpp:28-284, src/ode.cpp:20-174,
// src/ran2.cpp:13-32, src/static_ic.cpp:24-161) operation for operation, because the device
// step must start from bit-identical inputs.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "r3d_gpu.h"

namespace r3db {

// Values the reference derives from Params (include/params.hpp:125-145, src/params.cpp:14-66).
// Literals that the Fortran original wrote in single precision are float-rounded then widened.
struct Derived {
    int npx, npy, npz;
    int64_t nx, ny, nz;  // global extents with one ghost layer per side
    double c13, c23, c43;
    double gam[3], zeta[3];  // zeta[0] unused
    double hx, h2x, hy, h2y, hz, h2z;
    double repr, ore, cv, ocv, rkapst, orm, obeta, omx, omz;
};

Derived derive(const r3d_params& p);

// Throws std::invalid_argument with the reason when p is unsupported.
void check_params(const r3d_params& p);

// One grid line: physical coordinate, first and second derivative of the computational
// coordinate, and the spacing used by the dt limiter.
struct Line {
    std::vector<double> s, d1, d2, dd;
};
struct Metrics {
    Line x, y, z;
    std::vector<double> rkapa, dkapa;  // conductivity profile over z
};

// MKGRID (src/grid.cpp:28-146): maps scode in [0,1] to (sphys, dsds, d2sds2) along axis 1..3.
void map_coordinate(const r3d_params& p, double scode, int axis, double& sphys, double& dsds,
                    double& d2sds2);
Metrics build_metrics(const r3d_params& p, const Derived& d);

// RAN2 generator (Numerical Recipes), seeded by idum < 0.
class Ran2 {
   public:
    explicit Ran2(int idum) : idum_(idum) {}
    double next();

   private:
    int idum_;
    int iy_ = 0;
    int table_[97] = {0};
};

// Static polytrope by Bulirsch-Stoer integration, T(k), R(k) for k = 0..npz-1.
void static_profile(const r3d_params& p, std::vector<double>& t, std::vector<double>& r);

// The parts of the initial condition (src/static_ic.cpp:24-161) on global planes z0 .. z0+nz+1
// (the whole domain: z0 = 0, nz = npz), local plane k = global plane z0+k:
//  * columns: t[k], r[k] the static T and rho of the plane (interior cells; ghost planes: the
//    top T(0), R(0) and the bottom tb, rb), bfac[k] the magnetic layer's Bx (0 without LMAG and
//    on the ghost planes), tb;
//  * the metric lines into st's line arrays (x/y whole, z from global index z0, nz+2 entries);
//  * the perturbation draws: the RAN2 stream in the reference's global (k, j, i) order, one
//    interior plane at a time (a slab skips the draws of the planes above it).
struct IcColumns {
    std::vector<double> t, r, bfac;
    double tb = 1.0, rb = 1.0;
};
IcColumns ic_columns(const r3d_params& p, int z0, int nz);
void setup_lines(const r3d_params& p, const r3d_host_state& st, int z0, int nz);
class PerturbationDraws {
   public:
    PerturbationDraws(const r3d_params& p, int z0, int nz);
    // local planes [first, last] that carry the perturbation (empty when ampt == 0)
    int64_t first() const { return first_; }
    int64_t last() const { return last_; }
    // the npx*npy draws of the next plane, (j, i) order, into out
    void next_plane(double* out);

   private:
    Ran2 rng_;
    int64_t per_plane_, first_, last_;
};

// Fill st (arrays sized by the caller) with metrics, conductivity, the static IC, the seeded
// temperature perturbation and the periodic ghosts; returns tb in sc.
void setup_state(const r3d_params& p, const r3d_host_state& st, r3d_scalars& sc, int z0, int nz);

// Periodic x/y ghost copy of one field over every z plane (src/communicate.cpp:70-168 on one
// domain: y rows first, then x columns).
void fill_ghosts(double* f, int64_t nx, int64_t ny, int64_t nz);

}  // namespace r3db
