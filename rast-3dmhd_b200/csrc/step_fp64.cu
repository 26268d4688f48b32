// step_fp64.cu - the FP64 RK3 stage kernels (hydro; MHD adds the B fields).
//
// One launch per Wray stage computes, for every interior cell, the complete FLUXES right-hand
// side of src/fluxes.cpp:87-514 (+ the LMAG branch of golden/fortran/3dmhdsub.f:2146-2650 in
// step_mhd_fp64.cu) and applies the stage update of src/step.cpp:53-110 in its epilogue:
//     X' = Z + gam_s*dt*F            (Z = X at stage 1; the save_state copy is never made)
//     Z' = X' + zeta_{s+1}*dt*F      (stages 1 and 2; the reference's next mix_state)
// F is never stored.  The reference evaluates FLUXES as ~40 full-array sweeps with WW1..WW3
// temporaries; here every temporary is re-evaluated per cell with the literal expression the
// reference uses for it, and each accumulator (FU, FV, FW, FR, FT) receives its terms in the
// reference's order, so the result is bit-identical with FMA contraction off (-fmad=false).
//
// Tiling: a CTA owns a 32x8 column tile and marches down a chunk of z planes.  A three-plane
// ring in shared memory holds, with a one-cell x/y halo, the momenta, T, rho, 1/rho, the
// velocities and P = rho*T of planes k-1, k, k+1 (the 19-point stencil needs the twelve edge
// neighbours (i+-1,j+-1,k), (i+-1,j,k+-1), (i,j+-1,k+-1) of u, v, w).  1/rho and u,v,w are
// computed once per loaded cell.  Planes k = 1 and k = npz carry only the continuity flux
// (their momenta and T are rewritten by BCON, src/bcon.cpp:27-140, and the one-sided dRW/dz
// of src/fluxes.cpp:106-117 reaches two planes inward).  Ghost columns of X' are written by the
// owning thread, which replaces the periodic exchange of src/communicate.cpp:70-168.
//
// The third stage also evaluates, on the finished state, the per-cell time-step limits of the
// next step (src/step.cpp:122-229) and folds them into block minima; BCON does the same for
// the two boundary planes after rewriting them.
#include <cuda_runtime.h>

#include "r3d_device.cuh"
#include "r3d_kernels.h"

namespace r3dk {

constexpr int TX = 32, TY = 8, NT = TX * TY;
constexpr int SX = TX + 2, SY = TY + 2, SN = SX * SY;
enum { S_RU, S_RV, S_RW, S_TT, S_P, S_U, S_V, S_W, S_RO, S_RI, S_NF };
constexpr int kSlot = S_NF * SN;
constexpr size_t kStageSmem = 3 * kSlot * sizeof(double);

size_t stage_fp64_smem() { return kStageSmem; }

// Per-cell time-step limits (src/step.cpp:125-196): returns ww1, ww2, ww3 and the Mach term.
__device__ __forceinline__ void dt_terms(const Physics& ph, double ru, double rv, double rw,
                                         double ro, double tt, double b2sum, double dd,
                                         double rkap, double& w1, double& w2, double& w3,
                                         double& w4, double& um) {
    const double r = 1.0 / ro;
    double uu = (ru * ru + rv * rv + rw * rw) * r * r;
    um = ph.ogamma * uu / tt;
    if (ph.lmag) {
        const double b2 = b2sum * ph.obeta / ro;
        uu = uu + ph.gamma * tt + b2 + 2.0 * sqrt(uu * (ph.gamma * tt + b2));
        w4 = 0.5 * dd * dd * ph.rm;
    } else {
        uu = uu + ph.gamma * tt + 2.0 * sqrt(uu * ph.gamma * tt);
        w4 = 1e300;
    }
    w1 = dd / sqrt(uu);
    w2 = 0.5 * dd * dd * ph.repr * ph.cv * ro / rkap;
    w3 = 0.375 * dd * dd * ph.re * ro;
}

__device__ __forceinline__ double min_of3(double a, double b, double c) {
    const double m = (b < a) ? b : a;  // std::min(std::min(a, b), c)
    return (c < m) ? c : m;
}
__device__ __forceinline__ double fold_min(double acc, double v) { return (v < acc) ? v : acc; }
__device__ __forceinline__ double fold_max(double acc, double v) { return (acc < v) ? v : acc; }

// Block-wide fold of five running values and one atomic each into the device scalars.
__device__ void reduce_dt(double* red, double w1, double w2, double w3, double w4, double um,
                          Scalars* sc) {
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int nthr = blockDim.x * blockDim.y * blockDim.z;
    const int lane = tid & 31, warp = tid >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        w1 = fold_min(w1, __shfl_xor_sync(0xffffffffu, w1, o));
        w2 = fold_min(w2, __shfl_xor_sync(0xffffffffu, w2, o));
        w3 = fold_min(w3, __shfl_xor_sync(0xffffffffu, w3, o));
        w4 = fold_min(w4, __shfl_xor_sync(0xffffffffu, w4, o));
        um = fold_max(um, __shfl_xor_sync(0xffffffffu, um, o));
    }
    __syncthreads();
    if (lane == 0) {
        red[warp * 5 + 0] = w1;
        red[warp * 5 + 1] = w2;
        red[warp * 5 + 2] = w3;
        red[warp * 5 + 3] = w4;
        red[warp * 5 + 4] = um;
    }
    __syncthreads();
    if (tid == 0) {
        const int nw = (nthr + 31) / 32;
        for (int w = 1; w < nw; ++w) {
            w1 = fold_min(w1, red[w * 5 + 0]);
            w2 = fold_min(w2, red[w * 5 + 1]);
            w3 = fold_min(w3, red[w * 5 + 2]);
            w4 = fold_min(w4, red[w * 5 + 3]);
            um = fold_max(um, red[w * 5 + 4]);
        }
        atomicMin(&sc->wmin[0], order_key(w1));
        atomicMin(&sc->wmin[1], order_key(w2));
        atomicMin(&sc->wmin[2], order_key(w3));
        atomicMin(&sc->wmin[3], order_key(w4));
        atomicMax(&sc->umax, order_key(um));
    }
}

// Store v at (i,j) of plane base and at its periodic ghost images.
__device__ __forceinline__ void put_periodic(double* f, int64_t base, const Geometry& g, int i,
                                             int j, double v) {
    f[base + (int64_t)j * g.pitch + i] = v;
    const int gi = (i == 1) ? g.npx + 1 : ((i == g.npx) ? 0 : -1);
    const int gj = (j == 1) ? g.npy + 1 : ((j == g.npy) ? 0 : -1);
    if (gi >= 0) f[base + (int64_t)j * g.pitch + gi] = v;
    if (gj >= 0) f[base + (int64_t)gj * g.pitch + i] = v;
    if (gi >= 0 && gj >= 0) f[base + (int64_t)gj * g.pitch + gi] = v;
}

template <int STAGE>
__global__ void __launch_bounds__(NT, 2)
    stage_hydro_fp64(Geometry g, Physics ph, Lines L, FieldSet fs, Scalars* sc, int kchunk) {
    extern __shared__ double sm[];
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const int i0 = 1 + blockIdx.x * TX, j0 = 1 + blockIdx.y * TY;
    const int kb = 1 + blockIdx.z * kchunk;
    const int ke = min(g.npz, kb + kchunk - 1);
    const int i = i0 + tx, j = j0 + ty;
    const bool active = (i <= g.npx) && (j <= g.npy);
    const double* __restrict__ xru = fs.xin[0];
    const double* __restrict__ xrv = fs.xin[1];
    const double* __restrict__ xrw = fs.xin[2];
    const double* __restrict__ xro = fs.xin[3];
    const double* __restrict__ xtt = fs.xin[4];

    auto load_plane = [&](int kk) {
        double* b = sm + (kk % 3) * kSlot;
        for (int c = tid; c < SN; c += NT) {
            const int cx = c % SX, cy = c / SX;
            const int gi = i0 - 1 + cx, gj = j0 - 1 + cy;
            if (gi <= g.npx + 1 && gj <= g.npy + 1) {
                const int64_t n = (int64_t)kk * g.plane + (int64_t)gj * g.pitch + gi;
                const double ru = xru[n], rv = xrv[n], rw = xrw[n], ro = xro[n], tt = xtt[n];
                const double ri = 1.0 / ro;  // src/fluxes.cpp:137
                b[S_RU * SN + c] = ru;
                b[S_RV * SN + c] = rv;
                b[S_RW * SN + c] = rw;
                b[S_TT * SN + c] = tt;
                b[S_P * SN + c] = ro * tt;  // src/fluxes.cpp:136
                b[S_U * SN + c] = ru * ri;  // src/fluxes.cpp:158-166
                b[S_V * SN + c] = rv * ri;
                b[S_W * SN + c] = rw * ri;
                b[S_RO * SN + c] = ro;
                b[S_RI * SN + c] = ri;
            }
        }
    };

    // running dt limits (stage 3 only)
    double m1 = 1e300, m2 = 1e300, m3 = 1e300, m4 = 1e300, mu = 0.0;
    const double dt = sc->dt;
    const double cg = ph.gam[STAGE] * dt;
    const double cz = (STAGE < 2) ? ph.zeta[STAGE + 1] * dt : 0.0;
    const double hx = ph.hx, h2x = ph.h2x, hy = ph.hy, hz = ph.hz;
    const double dx1 = active ? L.dxxdx[i] : 0.0, d2x = active ? L.d2xxdx2[i] : 0.0;
    const double dyj = active ? L.dyydy[j] : 0.0, tmpy = active ? L.tmpy[j] : 0.0;
    const double tmpy1 = active ? L.tmpy1[j] : 0.0, tmpy2 = active ? L.tmpy2[j] : 0.0;
    const int s0 = (ty + 1) * SX + (tx + 1);

    load_plane(kb - 1);
    load_plane(kb);
    for (int k = kb; k <= ke; ++k) {
        load_plane(k + 1);
        __syncthreads();
        if (active) {
            const double* cm = sm + ((k + 2) % 3) * kSlot;
            const double* c0 = sm + (k % 3) * kSlot;
            const double* cp = sm + ((k + 1) % 3) * kSlot;
#define Q(P, F, DX, DY) P[(F)*SN + s0 + (DY)*SX + (DX)]
            const double tmpz = L.tmpz[k];
            const int64_t nc = (int64_t)k * g.plane + (int64_t)j * g.pitch + i;

            // ---- continuity, src/fluxes.cpp:87-121 ----
            double fr = (Q(c0, S_RU, -1, 0) - Q(c0, S_RU, 1, 0)) * hx * dx1;
            fr -= (Q(c0, S_RV, 0, 1) - Q(c0, S_RV, 0, -1)) * tmpy;
            double dwz;
            if (k == 1)
                dwz = (4.0 * Q(cp, S_RW, 0, 0) - xrw[nc + 2 * g.plane]) * tmpz;
            else if (k == g.npz)
                dwz = (xrw[nc - 2 * g.plane] - 4.0 * Q(cm, S_RW, 0, 0)) * tmpz;
            else
                dwz = (Q(cp, S_RW, 0, 0) - Q(cm, S_RW, 0, 0)) * tmpz;
            fr -= dwz;

            double fu = 0.0, fv = 0.0, fw = 0.0, ft = 0.0;
            if (k != 1 && k != g.npz) {
                const double dzk = L.dzzdz[k], tmpz1 = L.tmpz1[k], tmpz2 = L.tmpz2[k];
                const double U0 = Q(c0, S_U, 0, 0), V0 = Q(c0, S_V, 0, 0), W0 = Q(c0, S_W, 0, 0);
                const double T0 = Q(c0, S_TT, 0, 0), ri = Q(c0, S_RI, 0, 0);
                const double Uxp = Q(c0, S_U, 1, 0), Uxm = Q(c0, S_U, -1, 0);
                const double Uyp = Q(c0, S_U, 0, 1), Uym = Q(c0, S_U, 0, -1);
                const double Uzp = Q(cp, S_U, 0, 0), Uzm = Q(cm, S_U, 0, 0);
                const double Vxp = Q(c0, S_V, 1, 0), Vxm = Q(c0, S_V, -1, 0);
                const double Vyp = Q(c0, S_V, 0, 1), Vym = Q(c0, S_V, 0, -1);
                const double Vzp = Q(cp, S_V, 0, 0), Vzm = Q(cm, S_V, 0, 0);
                const double Wxp = Q(c0, S_W, 1, 0), Wxm = Q(c0, S_W, -1, 0);
                const double Wyp = Q(c0, S_W, 0, 1), Wym = Q(c0, S_W, 0, -1);
                const double Wzp = Q(cp, S_W, 0, 0), Wzm = Q(cm, S_W, 0, 0);

                // ---- buoyancy and pressure, src/fluxes.cpp:126-152 ----
                fw = ph.grav * Q(c0, S_RO, 0, 0);
                fw -= (Q(cp, S_P, 0, 0) - Q(cm, S_P, 0, 0)) * tmpz;
                fv = (Q(c0, S_P, 0, -1) - Q(c0, S_P, 0, 1)) * tmpy;
                fu = (Q(c0, S_P, -1, 0) - Q(c0, S_P, 1, 0)) * hx * dx1;

                // ---- momentum advection, src/fluxes.cpp:171-224 ----
                fu -= (Q(c0, S_RU, 1, 0) * Uxp - Q(c0, S_RU, -1, 0) * Uxm) * hx * dx1;
                fu -= (Q(c0, S_RU, 0, 1) * Vyp - Q(c0, S_RU, 0, -1) * Vym) * tmpy;
                fu -= (Q(cp, S_RU, 0, 0) * Wzp - Q(cm, S_RU, 0, 0) * Wzm) * tmpz;
                fv -= (Q(c0, S_RV, 1, 0) * Uxp - Q(c0, S_RV, -1, 0) * Uxm) * hx * dx1;
                fv -= (Q(c0, S_RV, 0, 1) * Vyp - Q(c0, S_RV, 0, -1) * Vym) * tmpy;
                fv -= (Q(cp, S_RV, 0, 0) * Wzp - Q(cm, S_RV, 0, 0) * Wzm) * tmpz;
                fw -= (Q(c0, S_RW, 1, 0) * Uxp - Q(c0, S_RW, -1, 0) * Uxm) * hx * dx1;
                fw -= (Q(c0, S_RW, 0, 1) * Vyp - Q(c0, S_RW, 0, -1) * Vym) * tmpy;
                fw -= (Q(cp, S_RW, 0, 0) * Wzp - Q(cm, S_RW, 0, 0) * Wzm) * tmpz;

                // ---- energy advection, src/fluxes.cpp:229-243 ----
                const double Txp = Q(c0, S_TT, 1, 0), Txm = Q(c0, S_TT, -1, 0);
                const double Typ = Q(c0, S_TT, 0, 1), Tym = Q(c0, S_TT, 0, -1);
                const double Tzp = Q(cp, S_TT, 0, 0), Tzm = Q(cm, S_TT, 0, 0);
                ft = -1.0 * U0 * (Txp - Txm) * hx * dx1;
                ft -= V0 * (Typ - Tym) * tmpy;
                ft -= W0 * (Tzp - Tzm) * tmpz;

                // ---- thermal conduction, src/fluxes.cpp:246-276 ----
                const double td = ph.tdiff;
                if (ph.kappa_const) {  // rkapa == 1, dkapa == 0: x*1 == x, ft + (+-0) == ft
                    ft += ((Txp - Txm) * hx * d2x + (Txp - 2.0 * T0 + Txm) * h2x * dx1 * dx1) * ri * td;
                    ft += ((Typ - Tym) * tmpy1 + (Typ - 2.0 * T0 + Tym) * tmpy2) * ri * td;
                    ft += ((Tzp - Tzm) * tmpz1 + (Tzp - 2.0 * T0 + Tzm) * tmpz2) * ri * td;
                } else {
                    const double rk = L.rkapa[k], dk = L.dkapa[k];
                    ft += ((Txp - Txm) * hx * d2x + (Txp - 2.0 * T0 + Txm) * h2x * dx1 * dx1) * ri * td * rk;
                    ft += ((Typ - Tym) * tmpy1 + (Typ - 2.0 * T0 + Tym) * tmpy2) * ri * td * rk;
                    ft += ((Tzp - Tzm) * tmpz1 + (Tzp - 2.0 * T0 + Tzm) * tmpz2) * ri * td * rk;
                    ft += (Tzp - Tzm) * hz * dzk * ri * td * dk;
                }

                // ---- viscous momentum, src/fluxes.cpp:281-320 ----
                const double ore = ph.ore, c43 = ph.c43;
                fu += ore * (c43 * ((Uxp - Uxm) * hx * d2x + (Uxp - 2.0 * U0 + Uxm) * h2x * dx1 * dx1) +
                             (Uyp - Uym) * tmpy1 + (Uyp - 2.0 * U0 + Uym) * tmpy2 +
                             (Uzp - Uzm) * tmpz1 + (Uzp - 2.0 * U0 + Uzm) * tmpz2);
                fv += ore * (((Vxp - Vxm) * hx * d2x + (Vxp - 2.0 * V0 + Vxm) * h2x * dx1 * dx1) +
                             c43 * ((Vyp - Vym) * tmpy1 + (Vyp - 2.0 * V0 + Vym) * tmpy2) +
                             (Vzp - Vzm) * tmpz1 + (Vzp - 2.0 * V0 + Vzm) * tmpz2);
                fw += ore * (((Wxp - Wxm) * hx * d2x + (Wxp - 2.0 * W0 + Wxm) * h2x * dx1 * dx1) +
                             (Wyp - Wym) * tmpy1 + (Wyp - 2.0 * W0 + Wym) * tmpy2 +
                             c43 * ((Wzp - Wzm) * tmpz1 + (Wzp - 2.0 * W0 + Wzm) * tmpz2));

                // ---- viscous heating, p dV and cross terms, src/fluxes.cpp:327-514 ----
                const double ux = (Uxp - Uxm) * hx * dx1;  // WW1 = dU/dx (:331, :416)
                const double vx = (Vxp - Vxm) * hx * dx1;  // WW2 = dV/dx (:336)
                const double wx = (Wxp - Wxm) * hx * dx1;  // WW3 = dW/dx (:341, :505)
                const double uy = (Uyp - Uym) * hy * dyj;  // :382
                const double vy = (Vyp - Vym) * hy * dyj;  // :397
                const double wy = (Wyp - Wym) * hy * dyj;  // :476
                const double uz = (Uzp - Uzm) * hz * dzk;  // :464
                const double vz = (Vzp - Vzm) * hz * dzk;  // :469
                const double wz = (Wzp - Wzm) * hz * dzk;  // :423
                const double th = ph.theat, th43 = ph.theat43, t13 = ph.t13, ocv = ph.ocv;
                ft += (c43 * ux * ux + vx * vx + wx * wx) * ri * th;  // :349
                ft -= ocv * ux * T0;                                   // :357
                // dV/dx and dU/dx one row up/down (:367-374)
                const double vx_jp = (Q(c0, S_V, 1, 1) - Q(c0, S_V, -1, 1)) * hx * dx1;
                const double vx_jm = (Q(c0, S_V, 1, -1) - Q(c0, S_V, -1, -1)) * hx * dx1;
                const double ux_jp = (Q(c0, S_U, 1, 1) - Q(c0, S_U, -1, 1)) * hx * dx1;
                const double ux_jm = (Q(c0, S_U, 1, -1) - Q(c0, S_U, -1, -1)) * hx * dx1;
                fu += t13 * (vx_jp - vx_jm) * hy * dyj;
                fv += t13 * (ux_jp - ux_jm) * hy * dyj;
                ft += (uy * uy + 2.0 * uy * vx) * ri * th;         // :389
                ft += vy * vy * ri * th43;                          // :404
                ft -= ocv * vy * T0;                                // :409
                ft += (wz * wz - ux * wz - ux * vy - vy * wz) * ri * th43;  // :432
                ft -= ocv * wz * T0;                                // :440
                // dW/dz one column left/right and one row up/down (:449-456)
                const double wz_ip = (Q(cp, S_W, 1, 0) - Q(cm, S_W, 1, 0)) * hz * dzk;
                const double wz_im = (Q(cp, S_W, -1, 0) - Q(cm, S_W, -1, 0)) * hz * dzk;
                const double wz_jp = (Q(cp, S_W, 0, 1) - Q(cm, S_W, 0, 1)) * hz * dzk;
                const double wz_jm = (Q(cp, S_W, 0, -1) - Q(cm, S_W, 0, -1)) * hz * dzk;
                fu += t13 * (wz_ip - wz_im) * hx * dx1;
                fv += t13 * (wz_jp - wz_jm) * hy * dyj;
                ft += (uz * uz + vz * vz + wy * wy + 2.0 * vz * wy) * ri * th;  // :484
                // dU/dz left/right, dV/dz up/down (:496-498)
                const double uz_ip = (Q(cp, S_U, 1, 0) - Q(cm, S_U, 1, 0)) * hz * dzk;
                const double uz_im = (Q(cp, S_U, -1, 0) - Q(cm, S_U, -1, 0)) * hz * dzk;
                const double vz_jp = (Q(cp, S_V, 0, 1) - Q(cm, S_V, 0, 1)) * hz * dzk;
                const double vz_jm = (Q(cp, S_V, 0, -1) - Q(cm, S_V, 0, -1)) * hz * dzk;
                fw += t13 * ((uz_ip - uz_im) * hx * dx1 + (vz_jp - vz_jm) * hy * dyj);
                ft += 2.0 * uz * wx * ri * th;  // :513

                // ---- rotation, src/fluxes.cpp:519-533 ----
                if (ph.lrot) {
                    fu += ph.omz * Q(c0, S_RV, 0, 0);
                    fv += -ph.omz * Q(c0, S_RU, 0, 0) + ph.omx * Q(c0, S_RW, 0, 0);
                    fw += -ph.omx * Q(c0, S_RV, 0, 0);
                }
            }

            // ---- stage update, src/step.cpp:53-110 ----
            const double F[5] = {fu, fv, fw, fr, ft};
            const int sidx[5] = {S_RU, S_RV, S_RW, S_RO, S_TT};
            const int64_t base = (int64_t)k * g.plane;
            double xn[5];
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                const double zq = (STAGE == 0) ? Q(c0, sidx[q], 0, 0) : fs.z[q][nc];
                xn[q] = zq + cg * F[q];
                put_periodic(fs.xout[q], base, g, i, j, xn[q]);
                if (STAGE < 2) fs.z[q][nc] = xn[q] + cz * F[q];
            }
            if (STAGE == 2 && k != 1 && k != g.npz) {
                const double dd = min_of3(L.ddx[i], L.ddy[j], L.ddz[k]);
                double w1, w2, w3, w4, um;
                dt_terms(ph, xn[0], xn[1], xn[2], xn[3], xn[4], 0.0, dd, L.rkapa[k], w1, w2, w3,
                         w4, um);
                m1 = fold_min(m1, w1);
                m2 = fold_min(m2, w2);
                m3 = fold_min(m3, w3);
                mu = fold_max(mu, um);
            }
#undef Q
        }
        __syncthreads();
    }
    if (STAGE == 2) reduce_dt(sm, m1, m2, m3, m4, mu, sc);
}

template __global__ void stage_hydro_fp64<0>(Geometry, Physics, Lines, FieldSet, Scalars*, int);
template __global__ void stage_hydro_fp64<1>(Geometry, Physics, Lines, FieldSet, Scalars*, int);
template __global__ void stage_hydro_fp64<2>(Geometry, Physics, Lines, FieldSet, Scalars*, int);

cudaError_t launch_stage_fp64(int stage, const Geometry& g, const Physics& ph, const Lines& L,
                              const FieldSet& fs, Scalars* sc, int kchunk, cudaStream_t st) {
    static bool configured = false;
    if (!configured) {
        cudaFuncSetAttribute(stage_hydro_fp64<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kStageSmem);
        cudaFuncSetAttribute(stage_hydro_fp64<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kStageSmem);
        cudaFuncSetAttribute(stage_hydro_fp64<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kStageSmem);
        configured = true;
    }
    dim3 block(TX, TY, 1);
    dim3 grid((g.npx + TX - 1) / TX, (g.npy + TY - 1) / TY, (g.npz + kchunk - 1) / kchunk);
    switch (stage) {
        case 0: stage_hydro_fp64<0><<<grid, block, kStageSmem, st>>>(g, ph, L, fs, sc, kchunk); break;
        case 1: stage_hydro_fp64<1><<<grid, block, kStageSmem, st>>>(g, ph, L, fs, sc, kchunk); break;
        default: stage_hydro_fp64<2><<<grid, block, kStageSmem, st>>>(g, ph, L, fs, sc, kchunk); break;
    }
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------
// BCON (src/bcon.cpp:12-141) on planes 1 and npz, their ghost images, and (after the third
// stage) the time-step limits of those two planes.
// ---------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) bcon_kernel(Geometry g, Physics ph, Lines L, Boundary b,
                                                   FieldSet fs, Scalars* sc, int with_dt) {
    __shared__ double red[5 * 8];
    const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
    const bool active = (i <= g.npx) && (j <= g.npy);
    double m1 = 1e300, m2 = 1e300, m3 = 1e300, m4 = 1e300, mu = 0.0;
    if (active) {
        double* ru = fs.xout[0];
        double* rv = fs.xout[1];
        double* rw = fs.xout[2];
        double* ro = fs.xout[3];
        double* tt = fs.xout[4];
        const double c13 = ph.c13, c23 = ph.c23, c43 = ph.c43;
        const int64_t P = g.plane, row = (int64_t)j * g.pitch + i;
        // top, k = 1 (src/bcon.cpp:27-98)
        {
            const int64_t n = P + row;
            const double ro1 = ro[n], ro2 = ro[n + P], ro3 = ro[n + 2 * P];
            const double u = ro1 * (c43 * ru[n + P] / ro2 - c13 * ru[n + 2 * P] / ro3);
            const double v = ro1 * (c43 * rv[n + P] / ro2 - c13 * rv[n + 2 * P] / ro3);
            double t;
            switch (b.top_mode) {
                case 0: t = 1.0; break;
                case 1: t = c43 * tt[n + P] - c13 * tt[n + 2 * P] - c23 * b.dz_top * b.theta; break;
                case 2: t = 1.0 - (1.0 - b.tpr) * L.plume_x[i] / b.hh * L.plume_y[j] / b.hh; break;
                case 3:
                    t = c43 * tt[n + P] - c13 * tt[n + 2 * P] -
                        c23 * b.dz_top * (b.theta - (b.theta - b.tpr) * L.plume_x[i] / b.hh * L.plume_y[j] / b.hh);
                    break;
                default: t = (i <= b.half_nx) ? 1.0 - b.tp : 1.0; break;
            }
            put_periodic(ru, P, g, i, j, u);
            put_periodic(rv, P, g, i, j, v);
            put_periodic(rw, P, g, i, j, 0.0);
            put_periodic(tt, P, g, i, j, t);
            double b2 = 0.0;
            if (ph.lmag) {
                put_periodic(fs.xout[7], P, g, i, j, 0.0);
                const double bx = fs.xout[5][n], by = fs.xout[6][n];
                b2 = bx * bx + by * by + 0.0 * 0.0;
            }
            if (with_dt) {
                const double dd = min_of3(L.ddx[i], L.ddy[j], L.ddz[1]);
                double w1, w2, w3, w4, um;
                dt_terms(ph, u, v, 0.0, ro1, t, b2, dd, L.rkapa[1], w1, w2, w3, w4, um);
                m1 = fold_min(m1, w1); m2 = fold_min(m2, w2); m3 = fold_min(m3, w3);
                m4 = fold_min(m4, w4); mu = fold_max(mu, um);
            }
        }
        // bottom, k = npz (src/bcon.cpp:104-139)
        {
            const int64_t n = (int64_t)g.npz * P + row;
            const double ro1 = ro[n], ro2 = ro[n - P], ro3 = ro[n - 2 * P];
            const double u = ro1 * (c43 * ru[n - P] / ro2 - c13 * ru[n - 2 * P] / ro3);
            const double v = ro1 * (c43 * rv[n - P] / ro2 - c13 * rv[n - 2 * P] / ro3);
            double t;
            if (b.bottom_mode == 0)
                t = b.tb;
            else
                t = c43 * tt[n - P] - c13 * tt[n - 2 * P] + c23 * b.dz_bot * b.theta / L.rkapa[g.npz];
            const int64_t base = (int64_t)g.npz * P;
            put_periodic(ru, base, g, i, j, u);
            put_periodic(rv, base, g, i, j, v);
            put_periodic(rw, base, g, i, j, 0.0);
            put_periodic(tt, base, g, i, j, t);
            double b2 = 0.0;
            if (ph.lmag) {
                put_periodic(fs.xout[7], base, g, i, j, 0.0);
                const double bx = fs.xout[5][n], by = fs.xout[6][n];
                b2 = bx * bx + by * by + 0.0 * 0.0;
            }
            if (with_dt) {
                const double dd = min_of3(L.ddx[i], L.ddy[j], L.ddz[g.npz]);
                double w1, w2, w3, w4, um;
                dt_terms(ph, u, v, 0.0, ro1, t, b2, dd, L.rkapa[g.npz], w1, w2, w3, w4, um);
                m1 = fold_min(m1, w1); m2 = fold_min(m2, w2); m3 = fold_min(m3, w3);
                m4 = fold_min(m4, w4); mu = fold_max(mu, um);
            }
        }
    }
    if (with_dt) reduce_dt(red, m1, m2, m3, m4, mu, sc);
}

cudaError_t launch_bcon(const Geometry& g, const Physics& ph, const Lines& L, const Boundary& b,
                        const FieldSet& fs, Scalars* sc, int with_dt, cudaStream_t st) {
    dim3 block(32, 8, 1);
    dim3 grid((g.npx + 31) / 32, (g.npy + 7) / 8, 1);
    bcon_kernel<<<grid, block, 0, st>>>(g, ph, L, b, fs, sc, with_dt);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------
// Full-domain time-step limits of the current state (used after an upload, and after a
// partial step, to seed the reduction the next step starts from).
// ---------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) dt_full_kernel(Geometry g, Physics ph, Lines L,
                                                      FieldSet fs, Scalars* sc) {
    __shared__ double red[5 * 8];
    const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
    double m1 = 1e300, m2 = 1e300, m3 = 1e300, m4 = 1e300, mu = 0.0;
    if (i <= g.npx && j <= g.npy) {
        const double dxy = (L.ddy[j] < L.ddx[i]) ? L.ddy[j] : L.ddx[i];
        for (int k = 1 + blockIdx.z; k <= g.npz; k += gridDim.z) {
            const int64_t n = (int64_t)k * g.plane + (int64_t)j * g.pitch + i;
            double b2 = 0.0;
            if (ph.lmag) {
                const double bx = fs.xin[5][n], by = fs.xin[6][n], bz = fs.xin[7][n];
                b2 = bx * bx + by * by + bz * bz;
            }
            const double dd = (L.ddz[k] < dxy) ? L.ddz[k] : dxy;
            double w1, w2, w3, w4, um;
            dt_terms(ph, fs.xin[0][n], fs.xin[1][n], fs.xin[2][n], fs.xin[3][n], fs.xin[4][n], b2,
                     dd, L.rkapa[k], w1, w2, w3, w4, um);
            m1 = fold_min(m1, w1); m2 = fold_min(m2, w2); m3 = fold_min(m3, w3);
            m4 = fold_min(m4, w4); mu = fold_max(mu, um);
        }
    }
    reduce_dt(red, m1, m2, m3, m4, mu, sc);
}

cudaError_t launch_dt_full(const Geometry& g, const Physics& ph, const Lines& L,
                           const FieldSet& fs, Scalars* sc, cudaStream_t st) {
    dim3 block(32, 8, 1);
    dim3 grid((g.npx + 31) / 32, (g.npy + 7) / 8, (unsigned)min(g.npz, 64));
    dt_full_kernel<<<grid, block, 0, st>>>(g, ph, L, fs, sc);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------
// Scalar bookkeeping: dt = sff*min(...) and umach = sqrt(max(...)) at the start of a step
// (src/step.cpp:133-141, 224-229), and nit/timc/timt at its end (src/step.cpp:254-256).
// ---------------------------------------------------------------------------------------
__global__ void step_begin_kernel(Physics ph, Scalars* sc) {
    const double w0 = order_value(sc->wmin[0]), w1 = order_value(sc->wmin[1]);
    const double w2 = order_value(sc->wmin[2]), w3 = order_value(sc->wmin[3]);
    double m = (w1 < w0) ? w1 : w0;
    m = (w2 < m) ? w2 : m;
    if (ph.lmag) m = (w3 < m) ? w3 : m;
    sc->dt = ph.sff * m;
    sc->umach = sqrt(order_value(sc->umax));
    sc->wmin[0] = sc->wmin[1] = sc->wmin[2] = sc->wmin[3] = order_key(1e300);
    sc->umax = order_key(0.0);
}

__global__ void step_end_kernel(Scalars* sc) {
    sc->nit += 1;
    sc->timc += sc->dt;
    sc->timt = sc->timi + sc->timc;
}

__global__ void reset_reduction_kernel(Scalars* sc) {
    sc->wmin[0] = sc->wmin[1] = sc->wmin[2] = sc->wmin[3] = order_key(1e300);
    sc->umax = order_key(0.0);
}

cudaError_t launch_step_begin(const Physics& ph, Scalars* sc, cudaStream_t st) {
    step_begin_kernel<<<1, 1, 0, st>>>(ph, sc);
    return cudaGetLastError();
}
cudaError_t launch_step_end(Scalars* sc, cudaStream_t st) {
    step_end_kernel<<<1, 1, 0, st>>>(sc);
    return cudaGetLastError();
}
cudaError_t launch_reset_reduction(Scalars* sc, cudaStream_t st) {
    reset_reduction_kernel<<<1, 1, 0, st>>>(sc);
    return cudaGetLastError();
}

}  // namespace r3dk
