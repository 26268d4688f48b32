// r3d_device.cuh - device-side data shared by the step kernels.
//
// Layout in HBM: one array per field over the global domain with one ghost layer per side,
// element (i,j,k) at k*plane + j*pitch + i, i in [0, npx+1], j in [0, npy+1], k in [0, npz+1].
// The row pitch is padded to a multiple of 16 doubles (128 B) so every row starts on a
// 128-byte boundary; tiles that start at i = 32*t (the halo column of interior column 32*t+1)
// are aligned for coalesced and TMA access.
#pragma once

#include <cstdint>

namespace r3dk {

constexpr int kMaxFields = 8;  // ru rv rw ro tt bx by bz

// Everything a stage kernel needs besides the field pointers.  Host-computed products keep
// the reference association (e.g. tmpy[j] = hy*dyydy[j], src/fluxes.cpp:90).
struct Geometry {
    int npx, npy, npz;  // npz: planes held by this device (a z slab of the domain, or all of it)
    int64_t pitch;      // doubles per row
    int64_t plane;      // doubles per z plane
    int top_edge;       // local plane 1 is the domain's top plane (BCON, one-sided stencils)
    int bot_edge;       // local plane npz is the domain's bottom plane
    int tile_rows;      // rows of the FP64 stage kernel's column tiles (stage_fp64_rows)
};

struct Physics {
    double hx, h2x, hy, hz, h2y, h2z;
    double c13, c23, c43, ore, ocv, grav;
    double tdiff;    // ocv/repr                     (src/fluxes.cpp:247)
    double theat;    // ocv*ore                      (src/fluxes.cpp:344)
    double theat43;  // c43*ocv*ore                  (src/fluxes.cpp:399)
    double t13;      // c13*ore                      (src/fluxes.cpp:362)
    double omx, omz;
    double gamma, ogamma, re, repr, cv, rm, obeta, orm, sff;
    double tmag;     // obeta*orm*ocv                (3dmhdsub.f:2308)
    double gam[3], zeta[3];
    int lrot, lmag;
    int kappa_const;  // rkapa == 1 and dkapa == 0 on every plane (exact shortcut)
    // embedded heat loss (itcon 2, 3dmhdsub.f:1799-1821): FT -= heat_pre * (1/rho) * heat_x/HH
    // * heat_y/HH * heat_z/HH, heat_pre = TP*OCV (tc == 0) or TP*OCV*0.5*(1+tanh(..)) per step
    int heat_on, hh_one;  // hh_one: HH == 1, where x/HH == x (the divisions are skipped)
    int top_free;         // itcon 3: BCON leaves the top temperature; its flux is formed there
    double heat_pre, hh;
    // density diffusion (ID 1, 2; 3dmhdsub.f:1316-1386): FR += (d2x + d2y)(rho - rom) * dh_ore*wwz
    // + d2z(rho - rom) * dv_ore*wwz, rom the horizontal mean of rho per plane
    int id_mode;
    double id_dh, id_dv, id_dh_ore, id_dv_ore;  // DH, DV and DH*ORE, DV*ORE
    float gamma_f, ogamma_f, obeta_f;  // float copies for the estimates of the dt filter
};

// 1D metric tables (device pointers).
struct Lines {
    const double *dxxdx, *d2xxdx2, *ddx;                      // [npx+2]
    const double *dyydy, *d2yydy2, *tmpy, *tmpy1, *tmpy2, *ddy;  // [npy+2]
    const double *dzzdz, *d2zzdz2, *tmpz, *tmpz1, *tmpz2;     // [npz+2]
    const double *ddz, *rkapa, *dkapa;                        // [npz+2]
    const double *plume_x, *plume_y;                          // [npx+2], [npy+2]
    // embedded heat loss (itcon 2): exp(CLN*(x - xp)^2) etc. per line, CLN = f4(-4 ln 2)/HH/HH
    const double *heat_x, *heat_y, *heat_z;                   // [npx+2], [npy+2], [npz+2]
    // density diffusion: the horizontal mean of rho per plane of the stage's input (written by
    // plane_mean_kernel before each stage) and the vertical profile WWZ   [npz+2] each
    const double *rom, *wwz;
};

// Error codes stored in Scalars::err by kernels that abandon a bounded wait.
enum { kErrNone = 0, kErrTmaTimeout = 1 };

// Boundary set-up for the BCON kernel (src/bcon.cpp:12-141).
struct Boundary {
    int top_mode;     // 0 const T=1, 1 const flux, 2 plume T, 3 plume flux, 4 half-domain T,
                      // 5 free (itcon 3: T evolves with its own flux, 3dmhdsub.f:2807-2887)
    int bottom_mode;  // 0 const T=tb, 1 const flux
    double tpr, hh, theta, tp, dz_top, dz_bot, tb;
    int half_nx;      // NX/2 for ITCON 4
};

// Device-resident scalars and the running dt reduction (ordered-integer keys).
struct Scalars {
    double dt, timc, timt, timi, umach, tb;
    int nit;
    int err;  // nonzero: a kernel gave up on a bounded wait (code = kernel id)
    // Test hook (r3d_gpu_debug_tma_extra): bytes added to every expected TMA transaction of the
    // stage kernels, so that their bounded waits run out; 0 in every normal run.
    unsigned int tx_extra;
    unsigned long long wmin[4];  // keys of min(ww1), min(ww2), min(ww3), min(vv)
    unsigned long long umax;     // key of max(ogamma*uu/tt)
    double mass, energy;         // diagnostics (r3d_gpu_totals)
    // Threshold filter of the third stage's limits (fold_dt_filtered): on whole-domain handles,
    // cells whose estimated ww1 exceeds thr_w1 and whose Mach term is below thr_um skip the exact
    // evaluation.  step_begin sets the thresholds from the previous limits widened by
    // thr_margin; step_end sets refold when the filtered minimum/maximum fails the check, and
    // the limits are then evaluated again over the whole state.
    int thr_on;
    int thr_local;  // a slab: thresholds from its own limits (wloc, uloc), saved before they are
                    // combined with the other slabs' (the check at step_end is then per slab)
    int refold;
    int refolds;  // number of re-evaluations since the upload (diagnostic)
    double thr_margin;
    double thr_w1, thr_um;
    unsigned long long wloc[4], uloc;  // this slab's limit keys before the cross-slab reduction
};

// Total order on doubles as unsigned keys: key(a) < key(b) iff a < b (NaN excluded).
__host__ __device__ inline unsigned long long order_key(double x) {
    unsigned long long b;
#ifdef __CUDA_ARCH__
    b = (unsigned long long)__double_as_longlong(x);
#else
    __builtin_memcpy(&b, &x, 8);
#endif
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__host__ __device__ inline double order_value(unsigned long long k) {
    unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
#ifdef __CUDA_ARCH__
    return __longlong_as_double((long long)b);
#else
    double x;
    __builtin_memcpy(&x, &b, 8);
    return x;
#endif
}

}  // namespace r3dk
