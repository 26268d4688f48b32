// step_fp32.cu - the FP32-bulk RK3 stage kernel (hydro), on packed FP32 pairs.
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
// R*T' + rho'*T0 + rho'*T'.
//
// Pairs: each thread evaluates two x-adjacent cells at once with sm_100's packed FP32
// instructions (add/mul/fma.rn.f32x2), so one instruction advances both cells.  The tile is 32
// cells wide: 16 threads per row, each on cells (2p+1, 2p+2) of the halo row, whose x
// neighbours are the aligned pairs (2p, 2p+1) and (2p+2, 2p+3) of shared memory - one 8-byte
// load each.
//
// Stage update: X' = Z + gam*dt*F rounds once to FP32 (one FMA); the RK accumulator
// Z' = X' + zeta*dt*F is formed from the unrounded X' with an error-free correction (the
// rounding residual of X' is recovered exactly by FMAs and added back), so Z' has the accuracy
// of an FP64 accumulation without FP64 arithmetic.  BCON, the dt reduction and the time sum run
// in FP64 on full values (bcon_fp32.cu; the third stage's dt limits below).
//
// Pipeline: a 32 x TY tile per CTA marching down z, a 4-slot TMA ring of (36, TY+2, 1) float
// boxes (x extent padded to a 16-byte multiple) and a 4-slot ring of derived u, v, w, P'; the
// thread's own Z accumulators are prefetched into L2 one plane ahead and loaded at the start of
// their plane (504x504x512 on B200 at 1965 MHz: 8.83 -> 8.40 ms per step against holding the
// next plane's values in registers).
#include <cuda.h>
#include <cuda_runtime.h>

#include "r3d_kernels.h"
#include "stage_common.cuh"
#include "tma.cuh"

#ifndef R3D_F32_TY
#define R3D_F32_TY 8  // tile rows
#endif

namespace r3dk {

namespace {
constexpr int TX = 32, PXN = TX / 2;  // cells per tile row, thread pairs per row
constexpr int SX = TX + 2;            // halo row width in cells (34)
constexpr int BOXX = 36;              // TMA box width (36 floats = 144 B)
enum { R_RU, R_RV, R_RW, R_RO, R_TT, R_NF };
enum { D_U, D_V, D_W, D_P, D_NF };
constexpr int NRAW = 4, NDER = 4;

template <int TYV>
struct Shape32 {
    static constexpr int SY = TYV + 2;
    static constexpr int NT = PXN * TYV;
    static constexpr int RAWF = (BOXX * SY + 31) / 32 * 32;  // floats per raw field box (128 B multiple)
    static constexpr int DERF = SX * SY;                     // floats per derived field (even)
    static constexpr int RAW_SLOT = R_NF * RAWF, DER_SLOT = D_NF * DERF;
    static constexpr size_t raw_bytes = (size_t)NRAW * RAW_SLOT * sizeof(float);
    static constexpr size_t der_bytes = ((size_t)NDER * DER_SLOT * sizeof(float) + 127) / 128 * 128;
    static constexpr size_t smem = raw_bytes + der_bytes + 64;
    static constexpr uint32_t plane_tx = R_NF * BOXX * SY * sizeof(float);
    // resident CTAs per SM: four in the first two stages (<= 128 registers, no spills); three
    // in the third, whose dt epilogue needs about 160 registers (measured at 504x504x512:
    // 4/4/3 2.889 ms per stage launch, 3/3/3 2.913, 4/4/4 with spills 3.070)
    static constexpr int ctas = TYV <= 8 ? 4 : 2;
#ifndef R3D_F32_CTAS_S2
#define R3D_F32_CTAS_S2 3
#endif
    static constexpr int ctas_s2 = TYV <= 8 ? R3D_F32_CTAS_S2 : 2;
    static constexpr int npairs = (SX / 2) * SY;    // derived pairs per plane
    static_assert(raw_bytes % 128 == 0 && (RAWF * 4) % 128 == 0, "TMA destinations stay 128-byte aligned");
    static_assert(DERF % 2 == 0 && SX % 2 == 0, "derived rows hold whole 8-byte pairs");
    static_assert(ctas * (smem + 1024) <= 228 * 1024, "resident CTAs per SM");
};
using Sh = Shape32<R3D_F32_TY>;

// packed FP32 arithmetic (one f32x2 instruction each)
typedef float2 v2;
__device__ __forceinline__ v2 B2(float a) { return make_float2(a, a); }
__device__ __forceinline__ v2 operator+(v2 a, v2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ v2 operator*(v2 a, v2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ v2 operator-(v2 a, v2 b) { return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a); }
__device__ __forceinline__ v2 fma2(v2 a, v2 b, v2 c) { return __ffma2_rn(a, b, c); }  // a*b + c
__device__ __forceinline__ v2 ld2(const float* p) { return *reinterpret_cast<const float2*>(p); }
__device__ __forceinline__ v2 mid(v2 a, v2 b) { return make_float2(a.y, b.x); }  // centre of (a, b)

// x stencil of one row of a field around the thread's pair: m = (f[c-1], f[c]), p = (f[c+1],
// f[c+2]) for cells (c, c+1) = (2p+1, 2p+2); c = (f[c], f[c+1])
struct Xs {
    v2 m, p;
    __device__ __forceinline__ v2 c() const { return mid(m, p); }
};
}  // namespace

void stage_fp32_box(unsigned* bx, unsigned* by) {
    *bx = BOXX;
    *by = Sh::SY;
}
int stage_fp32_ctas_per_sm() { return Sh::ctas; }

template <int STAGE>
__global__ void __launch_bounds__(Sh::NT, STAGE == 2 ? Sh::ctas_s2 : Sh::ctas)
    stage_fp32(const __grid_constant__ StageMaps maps, Geometry g, Physics ph, Lines L, Background bg,
               FieldSet32 fs, Scalars* sc, int kchunk) {
    constexpr int NT = Sh::NT, RAWF = Sh::RAWF, DERF = Sh::DERF;
    constexpr int RAW_SLOT = Sh::RAW_SLOT, DER_SLOT = Sh::DER_SLOT;
    extern __shared__ __align__(128) unsigned char smem[];
    float* raw = reinterpret_cast<float*>(smem);
    float* der = reinterpret_cast<float*>(smem + Sh::raw_bytes);
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + Sh::raw_bytes + Sh::der_bytes);
    __shared__ int s_abort;
    __shared__ double s_thr[2];  // third stage: thresholds of the dt filter (thr_w1, thr_um)

    const int tid = threadIdx.x;
    const int ty = tid / PXN, px = tid % PXN;
    const int i0 = 1 + blockIdx.x * TX, j0 = 1 + blockIdx.y * R3D_F32_TY;
    const int kb = 1 + blockIdx.z * kchunk;
    const int ke = min(g.npz, kb + kchunk - 1);
    const int i = i0 + 2 * px, j = j0 + ty;  // the pair's first cell
    const bool act0 = (i <= g.npx) && (j <= g.npy), act1 = (i + 1 <= g.npx) && (j <= g.npy);
    const int rrow = (ty + 1) * BOXX + 2 * px;  // raw offset of the aligned pair left of the cells
    const int drow = (ty + 1) * SX + 2 * px;    // derived offset, same
    int last_issued = kb - 2, last_waited = kb - 2;
    unsigned int tx_extra = 0;  // read by thread 0 (test hook, normally 0)

    auto issue = [&](int p) {
        last_issued = p;
        const int q = p - (kb - 1);
        uint64_t* bar = &bars[q % NRAW];
        float* dst = raw + (q % NRAW) * RAW_SLOT;
        mbar_expect_tx(bar, Sh::plane_tx + tx_extra);
#pragma unroll
        for (int f = 0; f < R_NF; ++f) tma_load_3d(dst + f * RAWF, &maps.m[f], bar, i0 - 1, j0 - 1, p);
    };
    // u, v, w, P' of every halo-tile cell of plane p, by aligned pairs (2q, 2q+1) of each row
    auto derive = [&](int p) -> bool {
        const int q = p - (kb - 1);
        if (!mbar_wait(&bars[q % NRAW], (q / NRAW) & 1)) return false;
        last_waited = p;
        const float* r = raw + (q % NRAW) * RAW_SLOT;
        float* d = der + (q % NDER) * DER_SLOT;
        const float R = bg.rf[p], T0 = bg.tf[p];
#pragma unroll
        for (int u = 0; u < (Sh::npairs + NT - 1) / NT; ++u) {
            const int c = tid + u * NT;
            if (c >= Sh::npairs) break;
            const int row = c / (SX / 2), col = 2 * (c % (SX / 2));
            const int rc = row * BOXX + col, dc = row * SX + col;
            const v2 rop = ld2(r + R_RO * RAWF + rc), ttp = ld2(r + R_TT * RAWF + rc);
            const v2 rho = B2(R) + rop;
            // hardware reciprocal (2 ulp): the stencils are FP32 anyway
            const v2 ri = make_float2(__fdividef(1.0f, rho.x), __fdividef(1.0f, rho.y));
            *reinterpret_cast<v2*>(d + D_U * DERF + dc) = ld2(r + R_RU * RAWF + rc) * ri;
            *reinterpret_cast<v2*>(d + D_V * DERF + dc) = ld2(r + R_RV * RAWF + rc) * ri;
            *reinterpret_cast<v2*>(d + D_W * DERF + dc) = ld2(r + R_RW * RAWF + rc) * ri;
            *reinterpret_cast<v2*>(d + D_P * DERF + dc) = fma2(B2(R), ttp, fma2(rop, B2(T0), rop * ttp));  // P - R*T0
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
    const v2 cg = B2((float)(ph.gam[STAGE] * dt));
    const v2 cz = B2((STAGE < 2) ? (float)(ph.zeta[STAGE + 1] * dt) : 0.0f);
    const int ia = act0 ? i : 1, ib = act1 ? i + 1 : ia, ja = act0 ? j : 1;
    const double dxy0 = (L.ddy[ja] < L.ddx[ia]) ? L.ddy[ja] : L.ddx[ia];  // the plane-independent part of dd
    const double dxy1 = (L.ddy[ja] < L.ddx[ib]) ? L.ddy[ja] : L.ddx[ib];
    const v2 cx = make_float2((float)(ph.hx * L.dxxdx[ia]), (float)(ph.hx * L.dxxdx[ib]));  // d/dx
    const v2 cx1 = make_float2((float)(ph.hx * L.d2xxdx2[ia]), (float)(ph.hx * L.d2xxdx2[ib]));
    const v2 cx2 = make_float2((float)(ph.h2x * L.dxxdx[ia] * L.dxxdx[ia]), (float)(ph.h2x * L.dxxdx[ib] * L.dxxdx[ib]));
    const v2 ncx = make_float2(-cx.x, -cx.y);
    const v2 cy = B2((float)L.tmpy[ja]), cy1 = B2((float)L.tmpy1[ja]), cy2 = B2((float)L.tmpy2[ja]);
    const v2 ncy = B2(-(float)L.tmpy[ja]);
    const v2 grav = B2((float)ph.grav), ore = B2((float)ph.ore), c43 = B2((float)ph.c43), c13o = B2((float)ph.t13);
    const v2 td = B2((float)ph.tdiff), th = B2((float)ph.theat), th43 = B2((float)ph.theat43), ocv = B2((float)ph.ocv);
    const v2 two = B2(2.0f), mtwo = B2(-2.0f);
    const float omx = (float)ph.omx, omz = (float)ph.omz;
    const int PL = (int)g.plane, PX = (int)g.pitch;
    const int col = ja * PX + ia;  // logical offset of the first cell in its plane
    const int gdy = (j == 1) ? g.npy * PX : ((j == g.npy) ? -g.npy * PX : 0);

    // the thread's Z accumulators (stored one column left, so the pair starts 8-byte aligned),
    // one plane ahead in registers
    v2 zc[5];

    for (int k = kb; k <= ke; ++k) {
        const int q = k - (kb - 1);
        if (STAGE > 0) {
            // this plane's accumulators (prefetched into L2 one plane earlier), issued before
            // the derive phase and the barrier; the next plane's, into L2
            const int n = k * PL + col - 1;
#pragma unroll
            for (int f = 0; f < 5; ++f) zc[f] = ld2(fs.z[f] + n);
            if (k < ke) {
#pragma unroll
                for (int f = 0; f < 5; ++f) prefetch_l2(fs.z[f] + n + PL);
            }
        }
        if (!derive(k + 1)) s_abort = 1;
        __syncthreads();
        if (s_abort) break;
        if (tid == 0) {
            fence_proxy_async();
            if (k + 2 <= ke + 1) issue(k + 2);
        }
        if (!act0) continue;
        const int nc = k * PL + col;
        const float* rm = raw + ((q + NRAW - 1) % NRAW) * RAW_SLOT;
        const float* r0 = raw + (q % NRAW) * RAW_SLOT;
        const float* rp = raw + ((q + 1) % NRAW) * RAW_SLOT;
        const float* dm = der + ((q + NDER - 1) % NDER) * DER_SLOT;
        const float* d0 = der + (q % NDER) * DER_SLOT;
        const float* dp = der + ((q + 1) % NDER) * DER_SLOT;
        // raw / derived field F of plane P at row offset DY: x stencil (Xs) or centre pair
#define RX_(P, F, DY) (Xs{ld2(P + (F)*RAWF + rrow + (DY)*BOXX), ld2(P + (F)*RAWF + rrow + (DY)*BOXX + 2)})
#define RC_(P, F, DY) make_float2(P[(F)*RAWF + rrow + (DY)*BOXX + 1], P[(F)*RAWF + rrow + (DY)*BOXX + 2])
#define DX_(P, F, DY) (Xs{ld2(P + (F)*DERF + drow + (DY)*SX), ld2(P + (F)*DERF + drow + (DY)*SX + 2)})
#define DC_(P, F, DY) make_float2(P[(F)*DERF + drow + (DY)*SX + 1], P[(F)*DERF + drow + (DY)*SX + 2])
        const float4 ka = bg.kf[3 * k], kb4 = bg.kf[3 * k + 1], kc4 = bg.kf[3 * k + 2];
        const v2 cz0 = B2(ka.x), ncz0 = B2(-ka.x);
        const bool edge = (k == 1 && g.top_edge) || (k == g.npz && g.bot_edge);

        const Xs RU = RX_(r0, R_RU, 0), RV = RX_(r0, R_RV, 0), RWx = RX_(r0, R_RW, 0);
        const v2 RUc = RU.c(), RVc = RV.c(), RWc = RWx.c();
        const v2 ROc = RC_(r0, R_RO, 0);
        // continuity (momenta only, no background)
        v2 fr = (RU.m - RU.p) * cx;
        fr = fma2(RC_(r0, R_RV, 1) - RC_(r0, R_RV, -1), ncy, fr);
        v2 dwz;
        if (k == 1 && g.top_edge)
            dwz = (B2(4.0f) * RC_(rp, R_RW, 0) - make_float2(fs.xin[R_RW][nc + 2 * PL], fs.xin[R_RW][nc + 2 * PL + 1])) * cz0;
        else if (k == g.npz && g.bot_edge)
            dwz = (make_float2(fs.xin[R_RW][nc - 2 * PL], fs.xin[R_RW][nc - 2 * PL + 1]) - B2(4.0f) * RC_(rm, R_RW, 0)) * cz0;
        else
            dwz = (RC_(rp, R_RW, 0) - RC_(rm, R_RW, 0)) * cz0;
        fr = fr - dwz;

        v2 fu = B2(0.f), fv = B2(0.f), fw = B2(0.f), ft = B2(0.f);
        if (!edge) {
            // every flux is a sum of independent terms, formed separately and added as a tree
            // (short dependency chains: FP32 carries no bit-exactness contract)
            const v2 cz1 = B2(ka.y), cz2 = B2(ka.z), czd = B2(ka.w);
            const Xs U = DX_(d0, D_U, 0), V = DX_(d0, D_V, 0), W = DX_(d0, D_W, 0);
            const v2 U0 = U.c(), V0 = V.c(), W0 = W.c();
            const v2 rho = B2(bg.rf[k]) + ROc;
            const v2 ri = make_float2(__fdividef(1.0f, rho.x), __fdividef(1.0f, rho.y));
            const Xs Uyp = DX_(d0, D_U, 1), Uym = DX_(d0, D_U, -1);
            const Xs Vyp = DX_(d0, D_V, 1), Vym = DX_(d0, D_V, -1);
            const v2 Uypc = Uyp.c(), Uymc = Uym.c(), Vypc = Vyp.c(), Vymc = Vym.c();
            const Xs Uzp = DX_(dp, D_U, 0), Uzm = DX_(dm, D_U, 0);
            const Xs Wzp = DX_(dp, D_W, 0), Wzm = DX_(dm, D_W, 0);
            const v2 Uzpc = Uzp.c(), Uzmc = Uzm.c(), Wzpc = Wzp.c(), Wzmc = Wzm.c();
            const v2 Vzp = DC_(dp, D_V, 0), Vzm = DC_(dm, D_V, 0);
            const v2 Wyp = DC_(d0, D_W, 1), Wym = DC_(d0, D_W, -1);

            // first differences and second-difference sums of the velocities
            const v2 dUx = U.p - U.m, dUy = Uypc - Uymc, dUz = Uzpc - Uzmc;
            const v2 dVx = V.p - V.m, dVy = Vypc - Vymc, dVz = Vzp - Vzm;
            const v2 dWx = W.p - W.m, dWy = Wyp - Wym, dWz = Wzpc - Wzmc;
            const v2 lUx = fma2(mtwo, U0, U.p) + U.m, lUy = fma2(mtwo, U0, Uypc) + Uymc, lUz = fma2(mtwo, U0, Uzpc) + Uzmc;
            const v2 lVx = fma2(mtwo, V0, V.p) + V.m, lVy = fma2(mtwo, V0, Vypc) + Vymc, lVz = fma2(mtwo, V0, Vzp) + Vzm;
            const v2 lWx = fma2(mtwo, W0, W.p) + W.m, lWy = fma2(mtwo, W0, Wyp) + Wym, lWz = fma2(mtwo, W0, Wzpc) + Wzmc;

            // pressure / buoyancy (hydrostatic background residual in FP64, deviations in FP32)
            const Xs P = DX_(d0, D_P, 0);
            const v2 pu = (P.m - P.p) * cx;
            const v2 pv = (DC_(d0, D_P, -1) - DC_(d0, D_P, 1)) * cy;
            const v2 pw = fma2(DC_(dp, D_P, 0) - DC_(dm, D_P, 0), ncz0, fma2(grav, ROc, B2(kb4.x)));

            // momentum advection, one term per direction
            const v2 RWzp = RC_(rp, R_RW, 0), RWzm = RC_(rm, R_RW, 0);
            const v2 au = fma2(RU.p * U.p - RU.m * U.m, ncx, (RC_(r0, R_RU, 1) * Vypc - RC_(r0, R_RU, -1) * Vymc) * ncy) +
                          (RC_(rp, R_RU, 0) * Wzpc - RC_(rm, R_RU, 0) * Wzmc) * ncz0;
            const v2 av = fma2(RV.p * U.p - RV.m * U.m, ncx, (RC_(r0, R_RV, 1) * Vypc - RC_(r0, R_RV, -1) * Vymc) * ncy) +
                          (RC_(rp, R_RV, 0) * Wzpc - RC_(rm, R_RV, 0) * Wzmc) * ncz0;
            const v2 aw = fma2(RWx.p * U.p - RWx.m * U.m, ncx, (RC_(r0, R_RW, 1) * Vypc - RC_(r0, R_RW, -1) * Vymc) * ncy) +
                          (RWzp * Wzpc - RWzm * Wzmc) * ncz0;

            // viscous momentum
            const v2 sux = fma2(dUx, cx1, lUx * cx2), suy = fma2(dUy, cy1, lUy * cy2), suz = fma2(dUz, cz1, lUz * cz2);
            const v2 svx = fma2(dVx, cx1, lVx * cx2), svy = fma2(dVy, cy1, lVy * cy2), svz = fma2(dVz, cz1, lVz * cz2);
            const v2 swx = fma2(dWx, cx1, lWx * cx2), swy = fma2(dWy, cy1, lWy * cy2), swz = fma2(dWz, cz1, lWz * cz2);
            const v2 vu = ore * fma2(c43, sux, suy + suz);
            const v2 vv = ore * fma2(c43, svy, svx + svz);
            const v2 vw = ore * fma2(c43, swz, swx + swy);

            // cross terms of the viscous stress
            const v2 vx_jp = (Vyp.p - Vyp.m) * cx, vx_jm = (Vym.p - Vym.m) * cx;
            const v2 ux_jp = (Uyp.p - Uyp.m) * cx, ux_jm = (Uym.p - Uym.m) * cx;
            const v2 wz_ip = (Wzp.p - Wzm.p) * czd, wz_im = (Wzp.m - Wzm.m) * czd;
            const v2 wz_jp = (DC_(dp, D_W, 1) - DC_(dm, D_W, 1)) * czd;
            const v2 wz_jm = (DC_(dp, D_W, -1) - DC_(dm, D_W, -1)) * czd;
            const v2 uz_ip = (Uzp.p - Uzm.p) * czd, uz_im = (Uzp.m - Uzm.m) * czd;
            const v2 vz_jp = (DC_(dp, D_V, 1) - DC_(dm, D_V, 1)) * czd;
            const v2 vz_jm = (DC_(dp, D_V, -1) - DC_(dm, D_V, -1)) * czd;
            const v2 xu = c13o * fma2(vx_jp - vx_jm, cy, (wz_ip - wz_im) * cx);
            const v2 xv = c13o * fma2(ux_jp - ux_jm, cy, (wz_jp - wz_jm) * cy);
            const v2 xw = c13o * fma2(uz_ip - uz_im, cx, (vz_jp - vz_jm) * cy);

            fu = (pu + au) + (vu + xu);
            fv = (pv + av) + (vv + xv);
            fw = (pw + aw) + (vw + xw);
            if (ph.lrot) {
                fu = fma2(B2(omz), RVc, fu);
                fv = fma2(B2(-omz), RUc, fma2(B2(omx), RWc, fv));
                fw = fma2(B2(-omx), RVc, fw);
            }

            // energy: advection and conduction on T = T0(k) + T', viscous heating, p dV
            const Xs T = RX_(r0, R_TT, 0);
            const v2 Tc = T.c();
            const v2 Typ = RC_(r0, R_TT, 1), Tym = RC_(r0, R_TT, -1);
            const v2 Tzp = RC_(rp, R_TT, 0), Tzm = RC_(rm, R_TT, 0);
            const v2 dTx = T.p - T.m, dTy = Typ - Tym, dTzd = Tzp - Tzm;
            const v2 dTz = B2(kb4.y) + dTzd;
            const v2 lTx = fma2(mtwo, Tc, T.p) + T.m;
            const v2 lTy = fma2(mtwo, Tc, Typ) + Tym;
            const v2 lTz = fma2(mtwo, Tc, Tzp) + Tzm;
            const v2 ea = fma2(U0 * dTx, ncx, (V0 * dTy) * ncy) + (W0 * dTz) * ncz0;
            const v2 lap = (fma2(dTx, cx1, lTx * cx2) + fma2(dTy, cy1, lTy * cy2)) +
                           (B2(kb4.z) + fma2(dTzd, cz1, lTz * cz2));
            const v2 ec = fma2(lap, td * B2(kb4.w), (dTz * czd) * (td * B2(kc4.x)));
            const v2 ux = dUx * cx, vx = dVx * cx, wx = dWx * cx;
            const v2 uy = dUy * cy, vy = dVy * cy, wy = dWy * cy;
            const v2 uz = dUz * czd, vz = dVz * czd, wz = dWz * czd;
            const v2 h1 = fma2(c43 * ux, ux, fma2(vx, vx, wx * wx)) + fma2(uy, uy, (two * uy) * vx);
            const v2 h2 = fma2(uz, uz, fma2(vz, vz, fma2(wy, wy, (two * vz) * wy))) + (two * uz) * wx;
            const v2 h3 = fma2(vy, vy, wz * wz) - fma2(ux, wz, fma2(ux, vy, vy * wz));
            const v2 eh = fma2(h1 + h2, th, h3 * th43);
            const v2 ep = (ocv * (B2(kc4.z) + Tc)) * ((ux + vy) + wz);
            ft = (ea + (ec + eh) * ri) - ep;
        }
        // stage update: X' = Z + cg*F (one rounding); Z' = (unrounded X') + cz*F through the
        // exact residual of X'
        const v2 F[5] = {fu, fv, fw, fr, ft};
        const v2 x0[5] = {RUc, RVc, RWc, ROc, RC_(r0, R_TT, 0)};
        v2 xn[5];
#pragma unroll
        for (int f = 0; f < 5; ++f) {
            const v2 zv = (STAGE == 0) ? x0[f] : zc[f];
            const v2 x = fma2(cg, F[f], zv);
            xn[f] = x;
            float* xo = fs.xout[f] + nc;
            xo[0] = x.x;
            if (act1) xo[1] = x.y;
            if (STAGE < 2) {
                const v2 r = fma2(cg, F[f], zv - x);  // (zv + cg*F) - x
                const v2 zz = x + fma2(cz, F[f], r);
                if (act1) *reinterpret_cast<v2*>(fs.z[f] + nc - 1) = zz;
                else fs.z[f][nc - 1] = zz.x;
            }
        }
        // periodic ghost images of the pair's cells on the domain's x/y faces
        const int gdx0 = (i == 1) ? g.npx : ((i == g.npx) ? -g.npx : 0);
        const int gdx1 = (i + 1 == g.npx) ? -g.npx : 0;
        if (gdx0 != 0 || gdy != 0 || (act1 && gdx1 != 0)) {
#pragma unroll
            for (int f = 0; f < 5; ++f) {
                float* xo = fs.xout[f] + nc;
                if (gdx0) xo[gdx0] = xn[f].x;
                if (gdy) xo[gdy] = xn[f].x;
                if (gdx0 && gdy) xo[gdx0 + gdy] = xn[f].x;
                if (act1) {
                    if (gdx1) xo[1 + gdx1] = xn[f].y;
                    if (gdy) xo[1 + gdy] = xn[f].y;
                    if (gdx1 && gdy) xo[1 + gdx1 + gdy] = xn[f].y;
                }
            }
        }
        if (STAGE == 2 && !edge) {  // dt limits, FP64 values on full state (filtered)
            const double rk = bg.r[k], tk = bg.t[k];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                if (h == 1 && !act1) break;
                const double dxy = h ? dxy1 : dxy0;
                const double dd = (L.ddz[k] < dxy) ? L.ddz[k] : dxy;  // min_of3(ddx, ddy, ddz)
                const float a0 = h ? xn[0].y : xn[0].x, a1 = h ? xn[1].y : xn[1].x, a2 = h ? xn[2].y : xn[2].x;
                const double ro = rk + (double)(h ? xn[3].y : xn[3].x), tt = tk + (double)(h ? xn[4].y : xn[4].x);
                if (ph.kappa_const)  // rkapa == 1 on every plane: x/rkapa == x, no division
                    fold_dt_filtered<true, false>(ph, a0, a1, a2, ro, tt, 0.0, dd, 1.0, s_thr[0], s_thr[1], m1,
                                                  m2, m3, m4, mu);
                else
                    fold_dt_filtered<false, false>(ph, a0, a1, a2, ro, tt, 0.0, dd, L.rkapa[k], s_thr[0],
                                                   s_thr[1], m1, m2, m3, m4, mu);
            }
        }
#undef RX_
#undef RC_
#undef DX_
#undef DC_
    }
    __syncthreads();
    if (s_abort) {
        if (tid == 0) {
            for (int p = last_waited + 1; p <= last_issued; ++p) {
                const int q = p - (kb - 1);
                (void)mbar_wait(&bars[q % NRAW], (q / NRAW) & 1);
            }
            atomicExch(&sc->err, kErrTmaTimeout);
        }
        return;
    }
    if (STAGE == 2) reduce_dt(reinterpret_cast<double*>(der), m1, m2, m3, m4, mu, sc);
}

cudaError_t launch_stage_fp32(int stage, const StageMaps& maps, const Geometry& g, const Physics& ph,
                              const Lines& L, const Background& bg, const FieldSet32& fs, Scalars* sc,
                              int kchunk, cudaStream_t st) {
    static bool configured = false;
    if (!configured) {
        cudaFuncSetAttribute(stage_fp32<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Sh::smem);
        cudaFuncSetAttribute(stage_fp32<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Sh::smem);
        cudaFuncSetAttribute(stage_fp32<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Sh::smem);
        // all of the unified L1 as shared memory, so that the resident CTAs fit
        cudaFuncSetAttribute(stage_fp32<0>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        cudaFuncSetAttribute(stage_fp32<1>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        cudaFuncSetAttribute(stage_fp32<2>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        configured = true;
    }
    dim3 block(Sh::NT, 1, 1);
    dim3 grid((g.npx + TX - 1) / TX, (g.npy + R3D_F32_TY - 1) / R3D_F32_TY, (g.npz + kchunk - 1) / kchunk);
    if (stage == 0) stage_fp32<0><<<grid, block, Sh::smem, st>>>(maps, g, ph, L, bg, fs, sc, kchunk);
    else if (stage == 1) stage_fp32<1><<<grid, block, Sh::smem, st>>>(maps, g, ph, L, bg, fs, sc, kchunk);
    else stage_fp32<2><<<grid, block, Sh::smem, st>>>(maps, g, ph, L, bg, fs, sc, kchunk);
    return cudaGetLastError();
}

}  // namespace r3dk
