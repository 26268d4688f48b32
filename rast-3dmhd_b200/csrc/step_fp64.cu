// step_fp64.cu - the fused FP64 RK3 stage kernel (hydro).
//
// One launch per Wray stage computes, for every interior cell, the complete FLUXES right-hand
// side of src/fluxes.cpp:87-514 and applies the stage update of src/step.cpp:53-110 in its
// epilogue:
//     X' = Z + gam_s*dt*F            (Z = X at stage 1; the save_state copy is never made)
//     Z' = X' + zeta_{s+1}*dt*F      (stages 1 and 2; the reference's next mix_state)
// F is never stored.  The reference evaluates FLUXES as ~40 full-array sweeps with WW1..WW3
// temporaries; here every temporary is re-evaluated per cell with the literal expression the
// reference uses for it, and each accumulator (FU, FV, FW, FR, FT) receives its terms in the
// reference's order, so with FMA contraction off (-fmad=false) the result is bit-identical.
//
// Pipeline: a CTA owns a 32x8 column tile and marches down a chunk of z planes.  Thread 0
// streams the five state fields of each plane, with a one-cell x/y halo, into a 4-slot ring
// by TMA (one 34x10x1 box per field, completion on a per-slot mbarrier), two planes ahead of
// the plane being computed.  Each loaded cell is then turned once into 1/rho, u, v, w and
// P = rho*T (src/fluxes.cpp:131-166) in a second 4-slot ring, so a single __syncthreads per
// plane orders everything: the plane k+1 derivation, the TMA refill of the slot of plane k-2,
// and the compute of plane k, which reads the 19-point stencil (the twelve edge neighbours of
// u, v, w come from the cross terms :367-374, :449-456, :496-498) from shared memory.
// Planes k = 1 and k = npz carry only the continuity flux: their momenta and T are rewritten
// by BCON (src/bcon.cpp:27-140) and the one-sided dRW/dz there (src/fluxes.cpp:106-117) reads
// two planes inward.  Ghost columns of X' are written by the owning thread (the periodic
// exchange of src/communicate.cpp:70-168).  The third stage also evaluates, on the finished
// state, the per-cell time-step limits of the next step (src/step.cpp:122-229).
#include <cuda.h>
#include <cuda_runtime.h>

#include "r3d_kernels.h"
#include "stage_common.cuh"
#include "tma.cuh"

namespace r3dk {

#ifndef R3D_STAGE_TY
#define R3D_STAGE_TY 8
#endif

namespace {
constexpr int TX = 32, TY = R3D_STAGE_TY, NT = TX * TY;
constexpr int kMinBlocks = (NT <= 256) ? 2 : 1;
constexpr int SX = TX + 2, SY = TY + 2, SN = SX * SY;  // 340 cells per halo tile
constexpr int RAWF = (SN + 15) / 16 * 16;   // doubles per raw field box, 128 B multiple
enum { R_RU, R_RV, R_RW, R_RO, R_TT, R_NF };
enum { D_U, D_V, D_W, D_P, D_RI, D_NF };
constexpr int NRAW = 4, NDER = 4;
constexpr int RAW_SLOT = R_NF * RAWF;      // doubles
constexpr int DER_SLOT = D_NF * SN;        // doubles
constexpr size_t kRawBytes = (size_t)NRAW * RAW_SLOT * sizeof(double);
constexpr size_t kDerBytes = (size_t)NDER * DER_SLOT * sizeof(double);
constexpr uint32_t kPlaneTx = R_NF * SN * sizeof(double);  // TMA bytes per plane
constexpr size_t kSmem = kRawBytes + kDerBytes + 64;
}  // namespace

size_t stage_fp64_smem() { return kSmem; }
void stage_fp64_box(unsigned* bx, unsigned* by) {
    *bx = SX;
    *by = SY;
}

template <int STAGE, bool KC>
__global__ void __launch_bounds__(NT, kMinBlocks)
    stage_hydro_fp64(const __grid_constant__ StageMaps maps, Geometry g, Physics ph, Lines L,
                     FieldSet fs, Scalars* sc, int kchunk) {
    extern __shared__ __align__(128) unsigned char smem[];
    double* raw = reinterpret_cast<double*>(smem);
    double* der = reinterpret_cast<double*>(smem + kRawBytes);
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kRawBytes + kDerBytes);
    __shared__ int s_abort;

    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const int i0 = 1 + blockIdx.x * TX, j0 = 1 + blockIdx.y * TY;
    const int kb = 1 + blockIdx.z * kchunk;
    const int ke = min(g.npz, kb + kchunk - 1);
    const int i = i0 + tx, j = j0 + ty;
    const bool active = (i <= g.npx) && (j <= g.npy);
    const int s0 = (ty + 1) * SX + (tx + 1);

    // plane p has local index q = p - (kb - 1); ring slot q % 4, mbarrier phase (q / 4) & 1
    int last_issued = kb - 2, last_waited = kb - 2;  // bookkeeping of thread 0 for the drain
    auto issue = [&](int p) {
        last_issued = p;
        const int q = p - (kb - 1);
        uint64_t* bar = &bars[q % NRAW];
        double* dst = raw + (q % NRAW) * RAW_SLOT;
        mbar_expect_tx(bar, kPlaneTx);
#pragma unroll
        for (int f = 0; f < R_NF; ++f) tma_load_3d(dst + f * RAWF, &maps.m[f], bar, i0 - 1, j0 - 1, p);
    };
    auto derive = [&](int p) -> bool {
        const int q = p - (kb - 1);
        if (!mbar_wait(&bars[q % NRAW], (q / NRAW) & 1)) return false;
        last_waited = p;
        const double* r = raw + (q % NRAW) * RAW_SLOT;
        double* d = der + (q % NDER) * DER_SLOT;
        for (int c = tid; c < SN; c += NT) {
            const double ro = r[R_RO * RAWF + c];
            const double ri = __drcp_rn(ro);  // == 1.0/ro, src/fluxes.cpp:137
            d[D_U * SN + c] = r[R_RU * RAWF + c] * ri;          // src/fluxes.cpp:158
            d[D_V * SN + c] = r[R_RV * RAWF + c] * ri;          // src/fluxes.cpp:162
            d[D_W * SN + c] = r[R_RW * RAWF + c] * ri;          // src/fluxes.cpp:166
            d[D_P * SN + c] = ro * r[R_TT * RAWF + c];          // src/fluxes.cpp:136
            d[D_RI * SN + c] = ri;
        }
        return true;
    };

    if (tid == 0) {
        // a CTA that finds an earlier timeout recorded leaves before issuing any copy
        s_abort = (*(volatile int*)&sc->err != kErrNone) ? 2 : 0;
        for (int b = 0; b < NRAW; ++b) mbar_init(&bars[b], 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (s_abort == 2) return;
    if (tid == 0) {
        issue(kb - 1);
        issue(kb);
        issue(kb + 1);
    }
    bool ok = derive(kb - 1);
    ok = derive(kb) && ok;
    if (!ok) s_abort = 1;

    double m1 = 1e300, m2 = 1e300, m3 = 1e300, m4 = 1e300, mu = 0.0;
    const double dt = sc->dt;
    const double cg = ph.gam[STAGE] * dt;
    const double cz = (STAGE < 2) ? ph.zeta[STAGE + 1] * dt : 0.0;
    const double hx = ph.hx, h2x = ph.h2x, hy = ph.hy, hz = ph.hz;
    const int ia = active ? i : 1, ja = active ? j : 1;
    const double dx1 = L.dxxdx[ia], d2x = L.d2xxdx2[ia];
    const double dyj = L.dyydy[ja], tmpy = L.tmpy[ja], tmpy1 = L.tmpy1[ja], tmpy2 = L.tmpy2[ja];

    // RK accumulator Z of the thread's own cell, loaded one plane ahead (registers)
    double zn[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    const int64_t col = (int64_t)ja * g.pitch + ia;
    if (STAGE > 0 && active) {
#pragma unroll
        for (int f = 0; f < 5; ++f) zn[f] = fs.z[f][(int64_t)kb * g.plane + col];
    }

    for (int k = kb; k <= ke; ++k) {
        const int q = k - (kb - 1);
        if (!derive(k + 1)) s_abort = 1;
        __syncthreads();
        if (s_abort) break;
        if (tid == 0 && k + 2 <= ke + 1) {
            fence_proxy_async();
            issue(k + 2);
        }
        double zq[5];
#pragma unroll
        for (int f = 0; f < 5; ++f) zq[f] = zn[f];
        if (STAGE > 0 && active && k < ke) {
#pragma unroll
            for (int f = 0; f < 5; ++f) zn[f] = fs.z[f][(int64_t)(k + 1) * g.plane + col];
        }
        if (active) {
            const int64_t nc = (int64_t)k * g.plane + col;
            const double* rm = raw + ((q + NRAW - 1) % NRAW) * RAW_SLOT;
            const double* r0 = raw + (q % NRAW) * RAW_SLOT;
            const double* rp = raw + ((q + 1) % NRAW) * RAW_SLOT;
            const double* dm = der + ((q + NDER - 1) % NDER) * DER_SLOT;
            const double* d0 = der + (q % NDER) * DER_SLOT;
            const double* dp = der + ((q + 1) % NDER) * DER_SLOT;
#define RW_(P, F, DX, DY) P[(F)*RAWF + s0 + (DY)*SX + (DX)]
#define DV_(P, F, DX, DY) P[(F)*SN + s0 + (DY)*SX + (DX)]
            const double tmpz = L.tmpz[k];

            // ---- continuity, src/fluxes.cpp:87-121 ----
            double fr = (RW_(r0, R_RU, -1, 0) - RW_(r0, R_RU, 1, 0)) * hx * dx1;
            fr -= (RW_(r0, R_RV, 0, 1) - RW_(r0, R_RV, 0, -1)) * tmpy;
            double dwz;
            if (k == 1)
                dwz = (4.0 * RW_(rp, R_RW, 0, 0) - fs.xin[2][nc + 2 * g.plane]) * tmpz;
            else if (k == g.npz)
                dwz = (fs.xin[2][nc - 2 * g.plane] - 4.0 * RW_(rm, R_RW, 0, 0)) * tmpz;
            else
                dwz = (RW_(rp, R_RW, 0, 0) - RW_(rm, R_RW, 0, 0)) * tmpz;
            fr -= dwz;

            double fu = 0.0, fv = 0.0, fw = 0.0, ft = 0.0;
            if (k != 1 && k != g.npz) {
                const double dzk = L.dzzdz[k], tmpz1 = L.tmpz1[k], tmpz2 = L.tmpz2[k];
                const double U0 = DV_(d0, D_U, 0, 0), V0 = DV_(d0, D_V, 0, 0), W0 = DV_(d0, D_W, 0, 0);
                const double T0 = RW_(r0, R_TT, 0, 0), ri = DV_(d0, D_RI, 0, 0);
                const double Uxp = DV_(d0, D_U, 1, 0), Uxm = DV_(d0, D_U, -1, 0);
                const double Uyp = DV_(d0, D_U, 0, 1), Uym = DV_(d0, D_U, 0, -1);
                const double Uzp = DV_(dp, D_U, 0, 0), Uzm = DV_(dm, D_U, 0, 0);
                const double Vxp = DV_(d0, D_V, 1, 0), Vxm = DV_(d0, D_V, -1, 0);
                const double Vyp = DV_(d0, D_V, 0, 1), Vym = DV_(d0, D_V, 0, -1);
                const double Vzp = DV_(dp, D_V, 0, 0), Vzm = DV_(dm, D_V, 0, 0);
                const double Wxp = DV_(d0, D_W, 1, 0), Wxm = DV_(d0, D_W, -1, 0);
                const double Wyp = DV_(d0, D_W, 0, 1), Wym = DV_(d0, D_W, 0, -1);
                const double Wzp = DV_(dp, D_W, 0, 0), Wzm = DV_(dm, D_W, 0, 0);

                // ---- buoyancy and pressure, src/fluxes.cpp:126-152 ----
                fw = ph.grav * RW_(r0, R_RO, 0, 0);
                fw -= (DV_(dp, D_P, 0, 0) - DV_(dm, D_P, 0, 0)) * tmpz;
                fv = (DV_(d0, D_P, 0, -1) - DV_(d0, D_P, 0, 1)) * tmpy;
                fu = (DV_(d0, D_P, -1, 0) - DV_(d0, D_P, 1, 0)) * hx * dx1;

                // ---- momentum advection, src/fluxes.cpp:171-224 ----
                fu -= (RW_(r0, R_RU, 1, 0) * Uxp - RW_(r0, R_RU, -1, 0) * Uxm) * hx * dx1;
                fu -= (RW_(r0, R_RU, 0, 1) * Vyp - RW_(r0, R_RU, 0, -1) * Vym) * tmpy;
                fu -= (RW_(rp, R_RU, 0, 0) * Wzp - RW_(rm, R_RU, 0, 0) * Wzm) * tmpz;
                fv -= (RW_(r0, R_RV, 1, 0) * Uxp - RW_(r0, R_RV, -1, 0) * Uxm) * hx * dx1;
                fv -= (RW_(r0, R_RV, 0, 1) * Vyp - RW_(r0, R_RV, 0, -1) * Vym) * tmpy;
                fv -= (RW_(rp, R_RV, 0, 0) * Wzp - RW_(rm, R_RV, 0, 0) * Wzm) * tmpz;
                fw -= (RW_(r0, R_RW, 1, 0) * Uxp - RW_(r0, R_RW, -1, 0) * Uxm) * hx * dx1;
                fw -= (RW_(r0, R_RW, 0, 1) * Vyp - RW_(r0, R_RW, 0, -1) * Vym) * tmpy;
                fw -= (RW_(rp, R_RW, 0, 0) * Wzp - RW_(rm, R_RW, 0, 0) * Wzm) * tmpz;

                // ---- energy advection, src/fluxes.cpp:229-243 ----
                const double Txp = RW_(r0, R_TT, 1, 0), Txm = RW_(r0, R_TT, -1, 0);
                const double Typ = RW_(r0, R_TT, 0, 1), Tym = RW_(r0, R_TT, 0, -1);
                const double Tzp = RW_(rp, R_TT, 0, 0), Tzm = RW_(rm, R_TT, 0, 0);
                ft = -1.0 * U0 * (Txp - Txm) * hx * dx1;
                ft -= V0 * (Typ - Tym) * tmpy;
                ft -= W0 * (Tzp - Tzm) * tmpz;

                // ---- thermal conduction, src/fluxes.cpp:246-276 ----
                const double td = ph.tdiff;
                if (KC) {  // rkapa == 1, dkapa == 0: x*1 == x, ft + (+-0) == ft
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
                const double vx_jp = (DV_(d0, D_V, 1, 1) - DV_(d0, D_V, -1, 1)) * hx * dx1;
                const double vx_jm = (DV_(d0, D_V, 1, -1) - DV_(d0, D_V, -1, -1)) * hx * dx1;
                const double ux_jp = (DV_(d0, D_U, 1, 1) - DV_(d0, D_U, -1, 1)) * hx * dx1;
                const double ux_jm = (DV_(d0, D_U, 1, -1) - DV_(d0, D_U, -1, -1)) * hx * dx1;
                fu += t13 * (vx_jp - vx_jm) * hy * dyj;
                fv += t13 * (ux_jp - ux_jm) * hy * dyj;
                ft += (uy * uy + 2.0 * uy * vx) * ri * th;                  // :389
                ft += vy * vy * ri * th43;                                   // :404
                ft -= ocv * vy * T0;                                         // :409
                ft += (wz * wz - ux * wz - ux * vy - vy * wz) * ri * th43;  // :432
                ft -= ocv * wz * T0;                                         // :440
                // dW/dz one column left/right and one row up/down (:449-456)
                const double wz_ip = (DV_(dp, D_W, 1, 0) - DV_(dm, D_W, 1, 0)) * hz * dzk;
                const double wz_im = (DV_(dp, D_W, -1, 0) - DV_(dm, D_W, -1, 0)) * hz * dzk;
                const double wz_jp = (DV_(dp, D_W, 0, 1) - DV_(dm, D_W, 0, 1)) * hz * dzk;
                const double wz_jm = (DV_(dp, D_W, 0, -1) - DV_(dm, D_W, 0, -1)) * hz * dzk;
                fu += t13 * (wz_ip - wz_im) * hx * dx1;
                fv += t13 * (wz_jp - wz_jm) * hy * dyj;
                ft += (uz * uz + vz * vz + wy * wy + 2.0 * vz * wy) * ri * th;  // :484
                // dU/dz left/right, dV/dz up/down (:496-498)
                const double uz_ip = (DV_(dp, D_U, 1, 0) - DV_(dm, D_U, 1, 0)) * hz * dzk;
                const double uz_im = (DV_(dp, D_U, -1, 0) - DV_(dm, D_U, -1, 0)) * hz * dzk;
                const double vz_jp = (DV_(dp, D_V, 0, 1) - DV_(dm, D_V, 0, 1)) * hz * dzk;
                const double vz_jm = (DV_(dp, D_V, 0, -1) - DV_(dm, D_V, 0, -1)) * hz * dzk;
                fw += t13 * ((uz_ip - uz_im) * hx * dx1 + (vz_jp - vz_jm) * hy * dyj);
                ft += 2.0 * uz * wx * ri * th;  // :513

                // ---- rotation, src/fluxes.cpp:519-533 ----
                if (ph.lrot) {
                    fu += ph.omz * RW_(r0, R_RV, 0, 0);
                    fv += -ph.omz * RW_(r0, R_RU, 0, 0) + ph.omx * RW_(r0, R_RW, 0, 0);
                    fw += -ph.omx * RW_(r0, R_RV, 0, 0);
                }
            }

            // ---- stage update, src/step.cpp:53-110 ----
            const double F[5] = {fu, fv, fw, fr, ft};
            const int64_t base = (int64_t)k * g.plane;
            double xn[5];
#pragma unroll
            for (int f = 0; f < 5; ++f) {
                const double zv = (STAGE == 0) ? RW_(r0, f, 0, 0) : zq[f];
                xn[f] = zv + cg * F[f];
                put_periodic(fs.xout[f], base, g, i, j, xn[f]);
                if (STAGE < 2) fs.z[f][nc] = xn[f] + cz * F[f];
            }
            if (STAGE == 2 && k != 1 && k != g.npz) {
                const double dd = min_of3(L.ddx[i], L.ddy[j], L.ddz[k]);
                double w1, w2, w3, w4, um;
                dt_terms<KC>(ph, xn[0], xn[1], xn[2], xn[3], xn[4], 0.0, dd, L.rkapa[k], w1, w2,
                             w3, w4, um);
                m1 = fold_min(m1, w1);
                m2 = fold_min(m2, w2);
                m3 = fold_min(m3, w3);
                mu = fold_max(mu, um);
            }
#undef RW_
#undef DV_
        }
    }
    __syncthreads();
    if (s_abort) {
        // a TMA wait timed out: drain our own copies (bounded), flag the error, leave
        if (tid == 0) {
            for (int p = last_waited + 1; p <= last_issued; ++p) {
                const int q = p - (kb - 1);
                (void)mbar_wait(&bars[q % NRAW], (q / NRAW) & 1);
            }
            atomicExch(&sc->err, kErrTmaTimeout);
        }
        return;
    }
    if (STAGE == 2) reduce_dt(der, m1, m2, m3, m4, mu, sc);
}

template <int STAGE, bool KC>
static void launch_one(dim3 grid, dim3 block, const StageMaps& maps, const Geometry& g,
                       const Physics& ph, const Lines& L, const FieldSet& fs, Scalars* sc,
                       int kchunk, cudaStream_t st) {
    static bool configured = false;
    if (!configured) {
        cudaFuncSetAttribute(stage_hydro_fp64<STAGE, KC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem);
        configured = true;
    }
    stage_hydro_fp64<STAGE, KC><<<grid, block, kSmem, st>>>(maps, g, ph, L, fs, sc, kchunk);
}

cudaError_t launch_stage_fp64(int stage, const StageMaps& maps, const Geometry& g,
                              const Physics& ph, const Lines& L, const FieldSet& fs, Scalars* sc,
                              int kchunk, cudaStream_t st) {
    dim3 block(TX, TY, 1);
    dim3 grid((g.npx + TX - 1) / TX, (g.npy + TY - 1) / TY, (g.npz + kchunk - 1) / kchunk);
    const bool kc = ph.kappa_const != 0;
    if (stage == 0) kc ? launch_one<0, true>(grid, block, maps, g, ph, L, fs, sc, kchunk, st)
                       : launch_one<0, false>(grid, block, maps, g, ph, L, fs, sc, kchunk, st);
    else if (stage == 1) kc ? launch_one<1, true>(grid, block, maps, g, ph, L, fs, sc, kchunk, st)
                            : launch_one<1, false>(grid, block, maps, g, ph, L, fs, sc, kchunk, st);
    else kc ? launch_one<2, true>(grid, block, maps, g, ph, L, fs, sc, kchunk, st)
            : launch_one<2, false>(grid, block, maps, g, ph, L, fs, sc, kchunk, st);
    return cudaGetLastError();
}

}  // namespace r3dk
