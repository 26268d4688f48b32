// step_fp32.cu - the FP32-bulk RK3 stage kernel (hydro).
//
// Storage: momenta ru, rv, rw and the deviations rho' = rho - R(k), T' = T - T0(k) from the
// static polytrope (R, T0 of src/ode.cpp:152-174, stitched over the global z index like the
// initial condition, src/static_ic.cpp:53-89) are stored in FP32, for X and for the RK
// accumulator Z: 20 B per cell per copy instead of 40.
//
// Arithmetic: the stencils of src/fluxes.cpp:87-533 are evaluated in FP32 (with FMA) on the
// deviations.  The background depends on z only, so every x/y difference of rho, T, P sees the
// deviation alone; every z term that involves the background is split into an FP64 per-plane
// part precomputed on the host and an FP32 deviation part:
//     g*rho - dP/dz          = hres(k) + g*rho' - dP'/dz,  hres(k) = g*R(k) - dP0/dz (FP64)
//     dT/dz, d2T/dz2 terms   = background difference (FP64) + deviation difference (FP32)
// so the near-hydrostatic cancellation in FW is never formed in single precision.  P' =
// R*T' + rho'*T0 + rho'*T'.  The stage accumulation X' = Z + gam*dt*F and Z' = X' + zeta*dt*F
// runs in FP64 on the FP32 inputs and rounds once on store; BCON, the dt reduction and the time
// sum run in FP64 on full values (bcon.cu).  The pipeline mirrors step_fp64.cu: a 32x8 tile
// per CTA marching down z, a 4-slot TMA ring of (36, 10, 1) float boxes (x extent padded to a
// 16-byte multiple) and a 4-slot ring of derived u, v, w, P', 1/rho.
#include <cuda.h>
#include <cuda_runtime.h>

#include "r3d_kernels.h"
#include "stage_common.cuh"
#include "tma.cuh"

namespace r3dk {

namespace {
constexpr int TX = 32, TY = 8, NT = TX * TY;
constexpr int SX = TX + 2, SY = TY + 2, SN = SX * SY;  // 340 halo cells used
constexpr int BOXX = 36;                               // TMA box width (36 floats = 144 B)
constexpr int RAWF = 384;                              // floats per raw field box (1536 B)
enum { R_RU, R_RV, R_RW, R_RO, R_TT, R_NF };
enum { D_U, D_V, D_W, D_P, D_RI, D_NF };
constexpr int NRAW = 4, NDER = 4, NZS = 3;
constexpr int RAW_SLOT = R_NF * RAWF;
constexpr int DER_SLOT = D_NF * SN;
constexpr int ZF = TX * TY;                // floats per Z box (no halo)
constexpr int Z_SLOT = 5 * ZF;
constexpr size_t kRawBytes = (size_t)NRAW * RAW_SLOT * sizeof(float);                   // 128 B multiple
constexpr size_t kDerBytes = ((size_t)NDER * DER_SLOT * sizeof(float) + 127) / 128 * 128;  // Z boxes 128 B aligned
constexpr size_t kZBytes = (size_t)NZS * Z_SLOT * sizeof(float);
constexpr uint32_t kPlaneTx = R_NF * BOXX * SY * sizeof(float);
constexpr uint32_t kZTx = 5 * ZF * sizeof(float);
constexpr size_t kSmem = kRawBytes + kDerBytes + kZBytes + 64;
static_assert(kRawBytes % 128 == 0 && (kRawBytes + kDerBytes) % 128 == 0 && (RAWF * 4) % 128 == 0 &&
                  (ZF * 4) % 128 == 0, "TMA destinations must stay 128-byte aligned");
static_assert(3 * (kSmem + 1024) <= 228 * 1024, "three CTAs per SM");
}  // namespace

void stage_fp32_box(unsigned* bx, unsigned* by) {
    *bx = BOXX;
    *by = SY;
}
void stage_fp32_zbox(unsigned* bx, unsigned* by) {
    *bx = TX;
    *by = TY;
}

template <int STAGE>
__global__ void __launch_bounds__(NT, 3)
    stage_fp32(const __grid_constant__ StageMaps maps, const __grid_constant__ StageMaps zmaps,
               Geometry g, Physics ph, Lines L, Background bg, FieldSet32 fs, Scalars* sc, int kchunk) {
    extern __shared__ __align__(128) unsigned char smem[];
    float* raw = reinterpret_cast<float*>(smem);
    float* der = reinterpret_cast<float*>(smem + kRawBytes);
    float* zsm = reinterpret_cast<float*>(smem + kRawBytes + kDerBytes);
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kRawBytes + kDerBytes + kZBytes);
    uint64_t* zbars = bars + NRAW;
    __shared__ int s_abort;
    __shared__ double s_thr[2];  // third stage: thresholds of the dt filter (thr_w1, thr_um)

    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const int i0 = 1 + blockIdx.x * TX, j0 = 1 + blockIdx.y * TY;
    const int kb = 1 + blockIdx.z * kchunk;
    const int ke = min(g.npz, kb + kchunk - 1);
    const int i = i0 + tx, j = j0 + ty;
    const bool active = (i <= g.npx) && (j <= g.npy);
    const int s0 = (ty + 1) * SX + (tx + 1);   // derived layout (34 wide)
    const int r0c = (ty + 1) * BOXX + (tx + 1);  // raw layout (36 wide)
    // the (at most two) halo cells this thread derives, as raw-box offsets
    const int rc0 = (tid / SX) * BOXX + (tid % SX);
    const int rc1 = ((tid + NT) / SX) * BOXX + ((tid + NT) % SX);

    int last_issued = kb - 2, last_waited = kb - 2;
    int zlast_issued = kb - 1, zlast_waited = kb - 1;
    // Z (the RK accumulator, stored one column left-shifted so interior boxes start 16-byte
    // aligned) of plane p, no halo, into a 3-slot ring; slot (p-kb)%3, phase ((p-kb)/3)&1
    unsigned int tx_extra = 0;  // read by thread 0 (test hook, normally 0)
    auto zissue = [&](int p) {
        zlast_issued = p;
        const int q = p - kb;
        uint64_t* bar = &zbars[q % NZS];
        float* dst = zsm + (q % NZS) * Z_SLOT;
        mbar_expect_tx(bar, kZTx + tx_extra);
#pragma unroll
        for (int f = 0; f < 5; ++f) tma_load_3d(dst + f * ZF, &zmaps.m[f], bar, i0 - 1, j0, p);
    };
    auto zwait = [&](int p) -> bool {
        const int q = p - kb;
        if (!mbar_wait(&zbars[q % NZS], (q / NZS) & 1)) return false;
        zlast_waited = p;
        return true;
    };
    auto issue = [&](int p) {
        last_issued = p;
        const int q = p - (kb - 1);
        uint64_t* bar = &bars[q % NRAW];
        float* dst = raw + (q % NRAW) * RAW_SLOT;
        mbar_expect_tx(bar, kPlaneTx + tx_extra);
#pragma unroll
        for (int f = 0; f < R_NF; ++f) tma_load_3d(dst + f * RAWF, &maps.m[f], bar, i0 - 1, j0 - 1, p);
    };
    auto derive = [&](int p) -> bool {
        const int q = p - (kb - 1);
        if (!mbar_wait(&bars[q % NRAW], (q / NRAW) & 1)) return false;
        last_waited = p;
        const float* r = raw + (q % NRAW) * RAW_SLOT;
        float* d = der + (q % NDER) * DER_SLOT;
        const float R = bg.rf[p], T0 = bg.tf[p];
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int c = tid + u * NT;
            if (c >= SN) break;
            const int rc = u == 0 ? rc0 : rc1;
            const float rop = r[R_RO * RAWF + rc], ttp = r[R_TT * RAWF + rc];
            const float ri = __fdividef(1.0f, R + rop);  // hardware reciprocal (2 ulp): the stencils are FP32 anyway
            d[D_U * SN + c] = r[R_RU * RAWF + rc] * ri;
            d[D_V * SN + c] = r[R_RV * RAWF + rc] * ri;
            d[D_W * SN + c] = r[R_RW * RAWF + rc] * ri;
            d[D_P * SN + c] = R * ttp + rop * T0 + rop * ttp;  // P' = P - R*T0
            d[D_RI * SN + c] = ri;
        }
        return true;
    };

    if (tid == 0) {
        s_abort = (*(volatile int*)&sc->err != kErrNone) ? 2 : 0;
        tx_extra = sc->tx_extra;
        if (STAGE == 2) {
            s_thr[0] = sc->thr_w1;
            s_thr[1] = sc->thr_um;
        }
        for (int b = 0; b < NRAW + NZS; ++b) mbar_init(&bars[b], 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (s_abort == 2) return;
    if (tid == 0) {
        issue(kb - 1);
        issue(kb);
        issue(kb + 1);
        if (STAGE > 0) {
            zissue(kb);
            if (kb + 1 <= ke) zissue(kb + 1);
        }
    }
    bool ok = derive(kb - 1);
    ok = derive(kb) && ok;
    if (!ok) s_abort = 1;

    double m1 = 1e300, m2 = 1e300, m3 = 1e300, m4 = 1e300, mu = 0.0;
    const double dt = sc->dt;
    const double cg = ph.gam[STAGE] * dt;
    const double cz = (STAGE < 2) ? ph.zeta[STAGE + 1] * dt : 0.0;
    const int ia = active ? i : 1, ja = active ? j : 1;
    const double dxy = (L.ddy[ja] < L.ddx[ia]) ? L.ddy[ja] : L.ddx[ia];  // the plane-independent part of dd
    const float cx = (float)(ph.hx * L.dxxdx[ia]);                       // d/dx
    const float cx1 = (float)(ph.hx * L.d2xxdx2[ia]);                    // second-derivative parts
    const float cx2 = (float)(ph.h2x * L.dxxdx[ia] * L.dxxdx[ia]);
    const float cy = (float)L.tmpy[ja], cy1 = (float)L.tmpy1[ja], cy2 = (float)L.tmpy2[ja];
    const float grav = (float)ph.grav, ore = (float)ph.ore, c43 = (float)ph.c43, c13o = (float)ph.t13;
    const float td = (float)ph.tdiff, th = (float)ph.theat, th43 = (float)ph.theat43, ocv = (float)ph.ocv;
    const float omx = (float)ph.omx, omz = (float)ph.omz;
    const int PL = (int)g.plane, PX = (int)g.pitch;
    const int col = ja * PX + ia;
    const int gdx = (i == 1) ? g.npx : ((i == g.npx) ? -g.npx : 0);
    const int gdy = (j == 1) ? g.npy * PX : ((j == g.npy) ? -g.npy * PX : 0);
    const bool ghost = active && (gdx != 0 || gdy != 0);


    for (int k = kb; k <= ke; ++k) {
        const int q = k - (kb - 1);
        if (!derive(k + 1)) s_abort = 1;
        __syncthreads();
        if (s_abort) break;
        if (tid == 0) {
            fence_proxy_async();
            if (k + 2 <= ke + 1) issue(k + 2);
            if (STAGE > 0 && k + 2 <= ke) zissue(k + 2);  // slot of plane k-1, free after the sync
        }
        const float* zt = zsm + ((k - kb) % NZS) * Z_SLOT;
        if (STAGE > 0 && !zwait(k)) s_abort = 1;
        if (!active) continue;
        const int nc = k * PL + col;
        const float* rm = raw + ((q + NRAW - 1) % NRAW) * RAW_SLOT;
        const float* r0 = raw + (q % NRAW) * RAW_SLOT;
        const float* rp = raw + ((q + 1) % NRAW) * RAW_SLOT;
        const float* dm = der + ((q + NDER - 1) % NDER) * DER_SLOT;
        const float* d0 = der + (q % NDER) * DER_SLOT;
        const float* dp = der + ((q + 1) % NDER) * DER_SLOT;
#define RW_(P, F, DX, DY) P[(F)*RAWF + r0c + (DY)*BOXX + (DX)]
#define DV_(P, F, DX, DY) P[(F)*SN + s0 + (DY)*SX + (DX)]
        const float4 ka = bg.kf[3 * k], kb4 = bg.kf[3 * k + 1], kc4 = bg.kf[3 * k + 2];
        const float cz0 = ka.x;
        const bool edge = (k == 1 && g.top_edge) || (k == g.npz && g.bot_edge);

        // continuity (momenta only, no background)
        float fr = (RW_(r0, R_RU, -1, 0) - RW_(r0, R_RU, 1, 0)) * cx;
        fr -= (RW_(r0, R_RV, 0, 1) - RW_(r0, R_RV, 0, -1)) * cy;
        float dwz;
        if (k == 1 && g.top_edge)
            dwz = (4.0f * RW_(rp, R_RW, 0, 0) - fs.xin[R_RW][nc + 2 * PL]) * cz0;
        else if (k == g.npz && g.bot_edge)
            dwz = (fs.xin[R_RW][nc - 2 * PL] - 4.0f * RW_(rm, R_RW, 0, 0)) * cz0;
        else
            dwz = (RW_(rp, R_RW, 0, 0) - RW_(rm, R_RW, 0, 0)) * cz0;
        fr -= dwz;

        float fu = 0.f, fv = 0.f, fw = 0.f, ft = 0.f;
        if (!edge) {
            const float cz1 = ka.y, cz2 = ka.z, czd = ka.w;
            const float U0 = DV_(d0, D_U, 0, 0), V0 = DV_(d0, D_V, 0, 0), W0 = DV_(d0, D_W, 0, 0);
            const float ri = DV_(d0, D_RI, 0, 0);
            const float T0 = kc4.z + RW_(r0, R_TT, 0, 0);  // full T
            const float Uxp = DV_(d0, D_U, 1, 0), Uxm = DV_(d0, D_U, -1, 0);
            const float Uyp = DV_(d0, D_U, 0, 1), Uym = DV_(d0, D_U, 0, -1);
            const float Uzp = DV_(dp, D_U, 0, 0), Uzm = DV_(dm, D_U, 0, 0);
            const float Vxp = DV_(d0, D_V, 1, 0), Vxm = DV_(d0, D_V, -1, 0);
            const float Vyp = DV_(d0, D_V, 0, 1), Vym = DV_(d0, D_V, 0, -1);
            const float Vzp = DV_(dp, D_V, 0, 0), Vzm = DV_(dm, D_V, 0, 0);
            const float Wxp = DV_(d0, D_W, 1, 0), Wxm = DV_(d0, D_W, -1, 0);
            const float Wyp = DV_(d0, D_W, 0, 1), Wym = DV_(d0, D_W, 0, -1);
            const float Wzp = DV_(dp, D_W, 0, 0), Wzm = DV_(dm, D_W, 0, 0);

            // buoyancy and pressure: hydrostatic background residual in FP64, deviations in FP32
            fw = kb4.x + grav * RW_(r0, R_RO, 0, 0) - (DV_(dp, D_P, 0, 0) - DV_(dm, D_P, 0, 0)) * cz0;
            fv = (DV_(d0, D_P, 0, -1) - DV_(d0, D_P, 0, 1)) * cy;
            fu = (DV_(d0, D_P, -1, 0) - DV_(d0, D_P, 1, 0)) * cx;

            // momentum advection
            fu -= (RW_(r0, R_RU, 1, 0) * Uxp - RW_(r0, R_RU, -1, 0) * Uxm) * cx;
            fu -= (RW_(r0, R_RU, 0, 1) * Vyp - RW_(r0, R_RU, 0, -1) * Vym) * cy;
            fu -= (RW_(rp, R_RU, 0, 0) * Wzp - RW_(rm, R_RU, 0, 0) * Wzm) * cz0;
            fv -= (RW_(r0, R_RV, 1, 0) * Uxp - RW_(r0, R_RV, -1, 0) * Uxm) * cx;
            fv -= (RW_(r0, R_RV, 0, 1) * Vyp - RW_(r0, R_RV, 0, -1) * Vym) * cy;
            fv -= (RW_(rp, R_RV, 0, 0) * Wzp - RW_(rm, R_RV, 0, 0) * Wzm) * cz0;
            fw -= (RW_(r0, R_RW, 1, 0) * Uxp - RW_(r0, R_RW, -1, 0) * Uxm) * cx;
            fw -= (RW_(r0, R_RW, 0, 1) * Vyp - RW_(r0, R_RW, 0, -1) * Vym) * cy;
            fw -= (RW_(rp, R_RW, 0, 0) * Wzp - RW_(rm, R_RW, 0, 0) * Wzm) * cz0;

            // energy advection and conduction on T = T0(k) + T'
            const float Tc = RW_(r0, R_TT, 0, 0);
            const float dTx = RW_(r0, R_TT, 1, 0) - RW_(r0, R_TT, -1, 0);
            const float dTy = RW_(r0, R_TT, 0, 1) - RW_(r0, R_TT, 0, -1);
            const float dTz = kb4.y + (RW_(rp, R_TT, 0, 0) - RW_(rm, R_TT, 0, 0));
            const float lTx = RW_(r0, R_TT, 1, 0) - 2.0f * Tc + RW_(r0, R_TT, -1, 0);
            const float lTy = RW_(r0, R_TT, 0, 1) - 2.0f * Tc + RW_(r0, R_TT, 0, -1);
            const float lTz = RW_(rp, R_TT, 0, 0) - 2.0f * Tc + RW_(rm, R_TT, 0, 0);
            ft = -U0 * dTx * cx - V0 * dTy * cy - W0 * dTz * cz0;
            const float lap = (dTx * cx1 + lTx * cx2) + (dTy * cy1 + lTy * cy2) +
                              (kb4.z + (RW_(rp, R_TT, 0, 0) - RW_(rm, R_TT, 0, 0)) * cz1 + lTz * cz2);
            ft += lap * ri * td * kb4.w + dTz * czd * ri * td * kc4.x;

            // viscous momentum
            fu += ore * (c43 * ((Uxp - Uxm) * cx1 + (Uxp - 2.0f * U0 + Uxm) * cx2) + (Uyp - Uym) * cy1 +
                         (Uyp - 2.0f * U0 + Uym) * cy2 + (Uzp - Uzm) * cz1 + (Uzp - 2.0f * U0 + Uzm) * cz2);
            fv += ore * (((Vxp - Vxm) * cx1 + (Vxp - 2.0f * V0 + Vxm) * cx2) +
                         c43 * ((Vyp - Vym) * cy1 + (Vyp - 2.0f * V0 + Vym) * cy2) + (Vzp - Vzm) * cz1 +
                         (Vzp - 2.0f * V0 + Vzm) * cz2);
            fw += ore * (((Wxp - Wxm) * cx1 + (Wxp - 2.0f * W0 + Wxm) * cx2) + (Wyp - Wym) * cy1 +
                         (Wyp - 2.0f * W0 + Wym) * cy2 + c43 * ((Wzp - Wzm) * cz1 + (Wzp - 2.0f * W0 + Wzm) * cz2));

            // viscous heating, p dV, cross terms
            const float ux = (Uxp - Uxm) * cx, vx = (Vxp - Vxm) * cx, wx = (Wxp - Wxm) * cx;
            const float uy = (Uyp - Uym) * cy, vy = (Vyp - Vym) * cy, wy = (Wyp - Wym) * cy;
            const float uz = (Uzp - Uzm) * czd, vz = (Vzp - Vzm) * czd, wz = (Wzp - Wzm) * czd;
            ft += (c43 * ux * ux + vx * vx + wx * wx) * ri * th;
            ft -= ocv * ux * T0;
            ft += (uy * uy + 2.0f * uy * vx) * ri * th;
            ft += vy * vy * ri * th43;
            ft -= ocv * vy * T0;
            ft += (wz * wz - ux * wz - ux * vy - vy * wz) * ri * th43;
            ft -= ocv * wz * T0;
            ft += (uz * uz + vz * vz + wy * wy + 2.0f * vz * wy) * ri * th;
            ft += 2.0f * uz * wx * ri * th;
            const float vx_jp = (DV_(d0, D_V, 1, 1) - DV_(d0, D_V, -1, 1)) * cx;
            const float vx_jm = (DV_(d0, D_V, 1, -1) - DV_(d0, D_V, -1, -1)) * cx;
            const float ux_jp = (DV_(d0, D_U, 1, 1) - DV_(d0, D_U, -1, 1)) * cx;
            const float ux_jm = (DV_(d0, D_U, 1, -1) - DV_(d0, D_U, -1, -1)) * cx;
            const float wz_ip = (DV_(dp, D_W, 1, 0) - DV_(dm, D_W, 1, 0)) * czd;
            const float wz_im = (DV_(dp, D_W, -1, 0) - DV_(dm, D_W, -1, 0)) * czd;
            const float wz_jp = (DV_(dp, D_W, 0, 1) - DV_(dm, D_W, 0, 1)) * czd;
            const float wz_jm = (DV_(dp, D_W, 0, -1) - DV_(dm, D_W, 0, -1)) * czd;
            const float uz_ip = (DV_(dp, D_U, 1, 0) - DV_(dm, D_U, 1, 0)) * czd;
            const float uz_im = (DV_(dp, D_U, -1, 0) - DV_(dm, D_U, -1, 0)) * czd;
            const float vz_jp = (DV_(dp, D_V, 0, 1) - DV_(dm, D_V, 0, 1)) * czd;
            const float vz_jm = (DV_(dp, D_V, 0, -1) - DV_(dm, D_V, 0, -1)) * czd;
            fu += c13o * ((vx_jp - vx_jm) * cy + (wz_ip - wz_im) * cx);
            fv += c13o * ((ux_jp - ux_jm) * cy + (wz_jp - wz_jm) * cy);
            fw += c13o * ((uz_ip - uz_im) * cx + (vz_jp - vz_jm) * cy);

            if (ph.lrot) {
                fu += omz * RW_(r0, R_RV, 0, 0);
                fv += -omz * RW_(r0, R_RU, 0, 0) + omx * RW_(r0, R_RW, 0, 0);
                fw += -omx * RW_(r0, R_RV, 0, 0);
            }
        }

        // stage update in FP64, one rounding on store
        const float F[5] = {fu, fv, fw, fr, ft};
        float xn[5];
#pragma unroll
        for (int f = 0; f < 5; ++f) {
            const double zv = (STAGE == 0) ? (double)RW_(r0, f, 0, 0) : (double)zt[f * ZF + tid];
            const double x = zv + cg * (double)F[f];
            xn[f] = (float)x;
            fs.xout[f][nc] = xn[f];
            if (STAGE < 2) fs.z[f][nc - 1] = (float)(x + cz * (double)F[f]);
        }
        if (ghost) {
#pragma unroll
            for (int f = 0; f < 5; ++f) {
                if (gdx) fs.xout[f][nc + gdx] = xn[f];
                if (gdy) fs.xout[f][nc + gdy] = xn[f];
                if (gdx && gdy) fs.xout[f][nc + gdx + gdy] = xn[f];
            }
        }
        if (STAGE == 2 && !edge) {  // dt limits, FP64 values on full state (filtered)
            const double dd = (L.ddz[k] < dxy) ? L.ddz[k] : dxy;  // min_of3(ddx, ddy, ddz)
            const double ro = bg.r[k] + (double)xn[3], tt = bg.t[k] + (double)xn[4];
            if (ph.kappa_const)  // rkapa == 1 on every plane: x/rkapa == x, no division
                fold_dt_filtered<true, false>(ph, xn[0], xn[1], xn[2], ro, tt, 0.0, dd, 1.0, s_thr[0],
                                              s_thr[1], m1, m2, m3, m4, mu);
            else
                fold_dt_filtered<false, false>(ph, xn[0], xn[1], xn[2], ro, tt, 0.0, dd, L.rkapa[k], s_thr[0],
                                               s_thr[1], m1, m2, m3, m4, mu);
        }
#undef RW_
#undef DV_
    }
    __syncthreads();
    if (s_abort) {
        if (tid == 0) {
            for (int p = last_waited + 1; p <= last_issued; ++p) {
                const int q = p - (kb - 1);
                (void)mbar_wait(&bars[q % NRAW], (q / NRAW) & 1);
            }
            for (int p = zlast_waited + 1; p <= zlast_issued; ++p) {
                const int q = p - kb;
                (void)mbar_wait(&zbars[q % NZS], (q / NZS) & 1);
            }
            atomicExch(&sc->err, kErrTmaTimeout);
        }
        return;
    }
    if (STAGE == 2) reduce_dt(reinterpret_cast<double*>(der), m1, m2, m3, m4, mu, sc);
}

cudaError_t launch_stage_fp32(int stage, const StageMaps& maps, const StageMaps& zmaps,
                              const Geometry& g, const Physics& ph, const Lines& L,
                              const Background& bg, const FieldSet32& fs, Scalars* sc, int kchunk,
                              cudaStream_t st) {
    static bool configured = false;
    if (!configured) {
        cudaFuncSetAttribute(stage_fp32<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem);
        cudaFuncSetAttribute(stage_fp32<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem);
        cudaFuncSetAttribute(stage_fp32<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem);
        configured = true;
    }
    dim3 block(TX, TY, 1);
    dim3 grid((g.npx + TX - 1) / TX, (g.npy + TY - 1) / TY, (g.npz + kchunk - 1) / kchunk);
    if (stage == 0) stage_fp32<0><<<grid, block, kSmem, st>>>(maps, zmaps, g, ph, L, bg, fs, sc, kchunk);
    else if (stage == 1) stage_fp32<1><<<grid, block, kSmem, st>>>(maps, zmaps, g, ph, L, bg, fs, sc, kchunk);
    else stage_fp32<2><<<grid, block, kSmem, st>>>(maps, zmaps, g, ph, L, bg, fs, sc, kchunk);
    return cudaGetLastError();
}

}  // namespace r3dk
