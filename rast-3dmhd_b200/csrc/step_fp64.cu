// step_fp64.cu - the fused FP64 RK3 stage kernel (hydro and MHD).
//
// One launch per Wray stage computes, for every interior cell, the complete FLUXES right-hand
// side of src/fluxes.cpp:87-533 (with MHD, also the LMAG branch of
// golden/fortran/3dmhdsub.f:2146-2650: Lorentz force, ohmic heating, induction and magnetic
// diffusion) and applies the stage update of src/step.cpp:53-110 (3dmhdsub.f:957-1177 for B)
// in its epilogue:
//     X' = Z + gam_s*dt*F            (Z = X at stage 1; the save_state copy is never made)
//     Z' = X' + zeta_{s+1}*dt*F      (stages 1 and 2; the reference's next mix_state)
// F is never stored.  The reference evaluates FLUXES as ~40 full-array sweeps (~80 with LMAG)
// with WW1..WW3 and RU..TT as temporaries; here every temporary is re-evaluated per cell with
// the literal expression the reference uses for it, and each accumulator (FU, FV, FW, FR, FT,
// and the B fluxes WW1..WW3) receives its terms in the reference's order, so with FMA
// contraction off (-fmad=false) the result is bit-identical.
//
// Pipeline: a CTA owns a 32 x TY column tile (TY = 8 hydro; 6, or 8 on small grids, with MHD)
// and marches down a chunk of z planes (depth chosen per handle on the host).  Thread 0
// streams the state fields of each plane, with a one-cell x/y halo, into a ring by TMA (one
// (34, TY+2, 1) box per field, completion on a per-slot mbarrier), two planes ahead of the
// plane being computed.  Each loaded cell is then turned once into u, v, w (and, with MHD,
// 1/rho and P = rho*T; src/fluxes.cpp:131-166) in a second, 4-slot ring, so a single
// __syncthreads per plane orders everything: the plane k+1 derivation, the TMA refill of the
// slot of plane k-2 (hydro: of plane k-1, whose values the threads hold), and the compute of
// plane k, which reads the 19-point stencil (the twelve edge neighbours of u, v, w come from
// the cross terms :367-374, :449-456, :496-498) from shared memory.  Hydro threads compute two
// adjacent rows each, 128-thread CTAs, three per SM; MHD threads one row.
// Planes k = 1 and k = npz carry only the continuity flux and, with MHD, the Bx/By fluxes:
// their momenta, T and Bz are rewritten by BCON (src/bcon.cpp:27-140); the one-sided
// z-derivatives there (src/fluxes.cpp:106-117, 3dmhdsub.f:2245-2259, 2468-2487, 2577-2596)
// reach up to three planes inward and read those planes from global memory.  Ghost columns
// of X' are written by the owning thread (the periodic exchange of src/communicate.cpp:
// 70-168).  The third stage also evaluates, on the finished state, the per-cell time-step
// limits of the next step (src/step.cpp:122-229).
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>

#include "r3d_kernels.h"
#include "stage_common.cuh"
#include "tma.cuh"

#ifndef R3D_STAGE_TY
#define R3D_STAGE_TY 8  // tile rows, hydro
#endif
// MHD tiles have 6 rows (two 192-thread CTAs per SM fit beside the 8-field rings) or, on grids
// too small to give every SM two CTAs, 8 rows (one 256-thread CTA per SM); Geometry::tile_rows
// holds the handle's choice.
#ifndef R3D_CPT_S0
#define R3D_CPT_S0 2
#endif
#ifndef R3D_CPT_S1
#define R3D_CPT_S1 2
#endif
#ifndef R3D_CPT_S2
#define R3D_CPT_S2 2
#endif

namespace r3dk {

namespace {
constexpr int TX = 32, SX = TX + 2;
enum { R_RU, R_RV, R_RW, R_RO, R_TT, R_BX, R_BY, R_BZ };
enum { D_U, D_V, D_W, D_P, D_RI, D_NF };
constexpr int NDER = 4;
#ifndef R3D_ZAHEAD
#define R3D_ZAHEAD 1  // planes by which the L2 prefetch of the accumulators runs ahead
#endif
// Hydro keeps a lean shared-memory layout, so that three 128-thread CTAs fit on an SM: a 3-slot
// raw ring (the thread's own values of plane k-1 are carried in registers), and u, v, w only in
// the derived ring (1/rho of the thread's own cells stays in registers; P = rho*T is formed
// where it is used, the product the reference stores).  MHD keeps the 4-slot raw ring and the
// derived u, v, w, P, 1/rho.  Both prefetch the RK accumulators of the next plane into L2 and
// load a plane's accumulators during the plane - hydro after its fluxes, just before the stage
// update, MHD before its derive phase - which takes fewer registers than holding the next
// plane's values in registers (hydro: 40, and no spills).  Measured on B200 at 1965 MHz:
// 504x504x512 hydro 15.45 -> 14.9 ms per step, 126x126x256 MHD 0.946 -> 0.901 ms (0.936 with
// the hydro placement); a prefetch two planes ahead was slower in every placement.
template <bool MHD>
struct Ring {
    static constexpr bool lean = !MHD;
    static constexpr int nraw = lean ? 3 : 4;
    static constexpr int nder_f = lean ? 3 : D_NF;  // derived fields per slot
};

// Cells per thread: a hydro thread computes CPT adjacent rows of its tile column, so each warp
// carries CPT independent stencil evaluations (and shares the y-neighbour loads between them).
// Two rows in all three stages (at three CTAs per SM; with one row, 256-thread CTAs, the third
// stage was 2.5% slower); an MHD cell already needs most of the register file, so MHD threads
// take one row.
// The right-hand side's variant of a plane: interior, or a domain edge (one-sided continuity
// and B stencils; the momentum and energy fluxes, which BCON rewrites, not formed) - or, with
// FULL, the top edge whose temperature BCON leaves alone (itcon 3): one-sided continuity and
// every momentum and energy flux formed as on an interior plane, as the reference does on its
// edge planes (src/fluxes.cpp loops over k1..k2).
template <bool B, bool FULL = false>
struct EdgeTag {
    static constexpr bool value = B;
    static constexpr bool full = FULL;
};

// xp - 2.0 * x0 + xm in the reference's rounding, rn(rn(xp - rn(2 * x0)) + xm), with one FP64
// operation fewer: 2 * x0 is exact (a power-of-two scaling, subnormals included), so
// rn(xp - rn(2 * x0)) == rn(xp - 2 * x0) == fma(-2, x0, xp) for every x0 whose double does not
// overflow (|x0| <= DBL_MAX / 2), zero signs and infinities included.
__device__ __forceinline__ double d2sum(double xp, double x0, double xm) {
    return __fma_rn(-2.0, x0, xp) + xm;
}

template <bool MHD, int TYV>
struct Shape {
    static constexpr int ty = TYV;  // tile rows
    static constexpr int sy = ty + 2, sn = SX * sy;                     // cells per halo tile
    static constexpr int rawf = (sn + 15) / 16 * 16;  // doubles per raw field box, 128 B multiple
    static constexpr int nf = MHD ? 8 : 5;                 // raw fields per plane
    static constexpr int raw_slot = nf * rawf;             // doubles
    static constexpr int der_slot = Ring<MHD>::nder_f * sn;  // doubles
    static constexpr size_t raw_bytes = (size_t)Ring<MHD>::nraw * raw_slot * sizeof(double);
    static constexpr size_t der_bytes = (size_t)NDER * der_slot * sizeof(double);
    static constexpr uint32_t plane_tx = nf * sn * sizeof(double);  // TMA bytes per plane
    static constexpr size_t smem = raw_bytes + der_bytes + 64;
    static constexpr int min_blocks = (smem * 2 <= 227 * 1024 && TX * ty <= 256) ? 2 : 1;
    // resident CTAs per SM of a 128-thread hydro CTA (two rows per thread)
    static constexpr int min_blocks_lean = (smem + 1024) * 3 <= 228 * 1024 ? 3 : min_blocks;
    static_assert(raw_bytes % 128 == 0 && (rawf * 8) % 128 == 0, "TMA destinations 128-byte aligned");
};

template <bool MHD, int STAGE, int TYV>
struct Cells {
    static constexpr int cpt = MHD ? 1 : (STAGE == 0 ? R3D_CPT_S0 : (STAGE == 1 ? R3D_CPT_S1 : R3D_CPT_S2));
    static constexpr int nt = TX * TYV / cpt;  // threads per CTA
    static constexpr int min_blocks =
        (!MHD && nt <= 128) ? Shape<MHD, TYV>::min_blocks_lean : Shape<MHD, TYV>::min_blocks;
    static_assert(TYV % cpt == 0, "tile rows must divide among the threads");
};
}  // namespace

size_t stage_fp64_smem() { return Shape<false, R3D_STAGE_TY>::smem; }
int stage_fp64_ctas_per_sm(int mhd, int rows) {
    if (!mhd) return std::min({Cells<false, 0, R3D_STAGE_TY>::min_blocks, Cells<false, 1, R3D_STAGE_TY>::min_blocks,
                               Cells<false, 2, R3D_STAGE_TY>::min_blocks});
    return rows == 6 ? Shape<true, 6>::min_blocks : Shape<true, 8>::min_blocks;
}
int stage_fp64_rows(int mhd, int npx, int npy, int nloc, int num_sms) {
    if (!mhd) return R3D_STAGE_TY;
    const long tiles6 = (long)((npx + TX - 1) / TX) * ((npy + 5) / 6);
    return tiles6 * ((nloc + 15) / 16) >= 2L * num_sms ? 6 : 8;
}
void stage_fp64_box(int rows, unsigned* bx, unsigned* by) {
    *bx = SX;
    *by = rows + 2;
}

// TF (hydro, itcon 3 only): the top plane's flux is formed as on an interior plane (EdgeTag);
// IDD (hydro, ID 1 or 2 only): the density diffusion is added to FR (itcon 3 then at run time)
template <int STAGE, bool KC, bool MHD, bool EMIT, int TYV, bool TF = false, bool IDD = false>
__global__ void __launch_bounds__(Cells<MHD, STAGE, TYV>::nt, Cells<MHD, STAGE, TYV>::min_blocks)
    stage_fp64(const __grid_constant__ StageMaps maps, Geometry g, Physics ph, Lines L,
               FieldSet fs, Scalars* sc, int kchunk) {
    using S = Shape<MHD, TYV>;
    constexpr int NF = S::nf;
    constexpr int TY = S::ty, SN = S::sn, RAWF = S::rawf;
    constexpr int CPT = Cells<MHD, STAGE, TYV>::cpt, NTH = Cells<MHD, STAGE, TYV>::nt;
    extern __shared__ __align__(128) unsigned char smem[];
    double* raw = reinterpret_cast<double*>(smem);
    double* der = reinterpret_cast<double*>(smem + S::raw_bytes);
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + S::raw_bytes + S::der_bytes);
    __shared__ int s_abort;
    __shared__ int s_filter;     // third stage: threshold-filtered dt fold (Scalars::thr_on)
    __shared__ double s_thr[2];  // its thresholds thr_w1, thr_um

    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const int i0 = 1 + blockIdx.x * TX, j0 = 1 + blockIdx.y * TY;
    const int kb = 1 + blockIdx.z * kchunk;
    const int ke = min(g.npz, kb + kchunk - 1);
    const int i = i0 + tx, jr = j0 + ty * CPT;  // the thread's column and first row

    constexpr bool LEAN = Ring<MHD>::lean;
    constexpr int NRAW = Ring<MHD>::nraw;
    // the thread's own cells in the halo tile (row c of the thread: halo row ty*CPT + c + 1)
    const int own0 = (ty * CPT + 1) * SX + tx + 1;
    // lean layout: 1/rho of the own cells of the plane derived last (rin) and of the plane
    // being computed (riq)
    double rin[CPT], riq[CPT];

    // plane p has local index q = p - (kb - 1); ring slot q % NRAW, mbarrier phase (q / NRAW) & 1
    int last_issued = kb - 2, last_waited = kb - 2;  // bookkeeping of thread 0 for the drain
    unsigned int tx_extra = 0;                          // read by thread 0 (test hook, normally 0)
    auto issue = [&](int p) {
        last_issued = p;
        const int q = p - (kb - 1);
        uint64_t* bar = &bars[q % NRAW];
        double* dst = raw + (q % NRAW) * S::raw_slot;
        mbar_expect_tx(bar, S::plane_tx + tx_extra);
#pragma unroll
        for (int f = 0; f < NF; ++f) tma_load_3d(dst + f * RAWF, &maps.m[f], bar, i0 - 1, j0 - 1, p);
    };
    auto derive = [&](int p) -> bool {
        const int q = p - (kb - 1);
        if (!mbar_wait(&bars[q % NRAW], (q / NRAW) & 1)) return false;
        last_waited = p;
        const double* r = raw + (q % NRAW) * S::raw_slot;
        double* d = der + (q % NDER) * S::der_slot;
        if constexpr (LEAN) {
            // every thread its own cells (keeping their 1/rho), then the halo ring of the tile:
            // the top and bottom halo rows, then the left and right halo columns
#pragma unroll
            for (int c = 0; c < CPT; ++c) {
                const int n = own0 + c * SX;
                const double ri = __drcp_rn(r[R_RO * RAWF + n]);  // == 1.0/ro, src/fluxes.cpp:137
                d[D_U * SN + n] = r[R_RU * RAWF + n] * ri;        // src/fluxes.cpp:158
                d[D_V * SN + n] = r[R_RV * RAWF + n] * ri;        // src/fluxes.cpp:162
                d[D_W * SN + n] = r[R_RW * RAWF + n] * ri;        // src/fluxes.cpp:166
                rin[c] = ri;
            }
            constexpr int NHALO = 2 * SX + 2 * TY;
            for (int h = tid; h < NHALO; h += NTH) {
                const int e = h - 2 * SX;
                const int n = (h < SX) ? h : ((h < 2 * SX) ? (TY + 1) * SX + (h - SX) : (1 + (e >> 1)) * SX + ((e & 1) ? SX - 1 : 0));
                const double ri = __drcp_rn(r[R_RO * RAWF + n]);
                d[D_U * SN + n] = r[R_RU * RAWF + n] * ri;
                d[D_V * SN + n] = r[R_RV * RAWF + n] * ri;
                d[D_W * SN + n] = r[R_RW * RAWF + n] * ri;
            }
        } else {
            for (int c = tid; c < SN; c += NTH) {
                const double ro = r[R_RO * RAWF + c];
                const double ri = __drcp_rn(ro);  // == 1.0/ro, src/fluxes.cpp:137
                d[D_U * SN + c] = r[R_RU * RAWF + c] * ri;          // src/fluxes.cpp:158
                d[D_V * SN + c] = r[R_RV * RAWF + c] * ri;          // src/fluxes.cpp:162
                d[D_W * SN + c] = r[R_RW * RAWF + c] * ri;          // src/fluxes.cpp:166
                d[D_P * SN + c] = ro * r[R_TT * RAWF + c];          // src/fluxes.cpp:136
                d[D_RI * SN + c] = ri;
            }
        }
        return true;
    };

    if (tid == 0) {
        // a CTA that finds an earlier timeout recorded leaves before issuing any copy
        s_abort = (*(volatile int*)&sc->err != kErrNone) ? 2 : 0;
        tx_extra = sc->tx_extra;
        if (STAGE == 2) {
            s_filter = sc->thr_on;
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
    // lean layout: the own cells' values of the plane above (the momenta, T, and P = rho*T in
    // the rho slot: the k-1 neighbours of the plane computed), carried in registers from plane
    // to plane
    double cm[CPT][5];
    if constexpr (LEAN) {
        if (ok) {
#pragma unroll
            for (int c = 0; c < CPT; ++c)
#pragma unroll
                for (int f = 0; f < 5; ++f) cm[c][f] = raw[f * RAWF + own0 + c * SX];  // slot 0: plane kb-1
#pragma unroll
            for (int c = 0; c < CPT; ++c) cm[c][R_RO] = cm[c][R_RO] * cm[c][R_TT];  // P of plane kb-1
        }
    }
    ok = derive(kb) && ok;
    if (!ok) s_abort = 1;

    double m1 = 1e300, m2 = 1e300, m3 = 1e300, m4 = 1e300, mu = 0.0;
    const double dt = sc->dt;
    const double cg = ph.gam[STAGE] * dt;
    const double cz = (STAGE < 2) ? ph.zeta[STAGE + 1] * dt : 0.0;
    const double hx = ph.hx, h2x = ph.h2x, hy = ph.hy, hz = ph.hz;
    const int ia = (i <= g.npx) ? i : 1;
    const double dx1 = L.dxxdx[ia], d2x = L.d2xxdx2[ia];
    // 32-bit element offsets (a field holds < 2^31 elements, checked at create)
    const int PL = (int)g.plane, PX = (int)g.pitch;
    // offsets from a cell to its periodic ghost images (0: none)
    const int gdx = (i == 1) ? g.npx : ((i == g.npx) ? -g.npx : 0);

    // per row c of the thread: activity, y metrics, column offset
    bool actv[CPT];
    int colv[CPT];
    double dxyv[CPT];  // third stage: min(ddx[i], ddy[j]), the plane-independent part of dd
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
        const int j = jr + c;
        actv[c] = (i <= g.npx) && (j <= g.npy);
        colv[c] = ((j <= g.npy) ? j : 1) * PX + ia;
        if (STAGE == 2) {
            const int ja = (j <= g.npy) ? j : 1;
            dxyv[c] = (L.ddy[ja] < L.ddx[ia]) ? L.ddy[ja] : L.ddx[ia];
        }
    }

    for (int k = kb; k <= ke; ++k) {
        const int q = k - (kb - 1);
        // the RK accumulators Z of the thread's cells: the next plane's into L2, this plane's
        // (zq) loaded below
        double zq[CPT][NF];
        if (STAGE > 0 && k + R3D_ZAHEAD <= ke) {
#pragma unroll
            for (int c = 0; c < CPT; ++c)
                if (actv[c]) {
#pragma unroll
                    for (int f = 0; f < NF; ++f) prefetch_l2(fs.z[f] + (k + R3D_ZAHEAD) * PL + colv[c]);
                }
        }
        if constexpr (LEAN) {
#pragma unroll
            for (int c = 0; c < CPT; ++c) riq[c] = rin[c];
        }
        if constexpr (!LEAN) {
            // MHD: this plane's accumulators, issued before the derive phase and the barrier
#pragma unroll
            for (int c = 0; c < CPT; ++c) {
#pragma unroll
                for (int f = 0; f < NF; ++f) zq[c][f] = 0.0;
                if (STAGE > 0 && actv[c]) {
#pragma unroll
                    for (int f = 0; f < NF; ++f) zq[c][f] = fs.z[f][k * PL + colv[c]];
                }
            }
        }
        if (!derive(k + 1)) s_abort = 1;
        __syncthreads();
        if (s_abort) break;
        if (tid == 0 && k + 2 <= ke + 1) {
            fence_proxy_async();
            issue(k + 2);
        }
        const double* rm = raw + ((q + NRAW - 1) % NRAW) * S::raw_slot;
        const double* r0 = raw + (q % NRAW) * S::raw_slot;
        const double* rp = raw + ((q + 1) % NRAW) * S::raw_slot;
        const double* dm = der + ((q + NDER - 1) % NDER) * S::der_slot;
        const double* d0 = der + (q % NDER) * S::der_slot;
        const double* dp = der + ((q + 1) % NDER) * S::der_slot;
#define RW_(P, F, DX, DY) P[(F)*RAWF + s0 + (DY)*SX + (DX)]
#define DV_(P, F, DX, DY) P[(F)*SN + s0 + (DY)*SX + (DX)]
// own-cell raw value of plane k-1; P = rho*T on planes k (with x/y offsets), k+1 and k-1
#define RM_(F) (LEAN ? cm[c][F] : RW_(rm, F, 0, 0))
#define P0_(DX, DY) (LEAN ? RW_(r0, R_RO, DX, DY) * RW_(r0, R_TT, DX, DY) : DV_(d0, D_P, DX, DY))
#define PP_ (LEAN ? RW_(rp, R_RO, 0, 0) * RW_(rp, R_TT, 0, 0) : DV_(dp, D_P, 0, 0))
#define PM_ (LEAN ? cm[c][R_RO] : DV_(dm, D_P, 0, 0))  // lean: cm[.][R_RO] carries P
        const double tmpz = L.tmpz[k];
        const bool edge = (k == 1 && g.top_edge) || (k == g.npz && g.bot_edge);
        // right-hand sides of the thread's cells: all rows first, so that their independent
        // stencil evaluations can interleave, then the stage updates and stores
        double Fc[CPT][NF];
        // the plane's edge status is uniform over the CTA: one straight-line copy of the stencil
        // per case, so that the rows' evaluations share basic blocks
        auto rhs = [&](auto edge_tag) {
          constexpr bool EDGE = decltype(edge_tag)::value;
          constexpr bool FULLTOP = decltype(edge_tag)::full;
#pragma unroll
          for (int c = 0; c < CPT; ++c) {
#pragma unroll
            for (int f = 0; f < NF; ++f) Fc[c][f] = 0.0;
            const int j = jr + c, ja = (j <= g.npy) ? j : 1;
            const int s0 = (ty * CPT + c + 1) * SX + (tx + 1);
            const int nc = k * PL + colv[c];
            const double dyj = L.dyydy[ja], tmpy = L.tmpy[ja], tmpy1 = L.tmpy1[ja], tmpy2 = L.tmpy2[ja];
            // inactive rows (beyond a ragged tile edge) compute on in-bounds data and are not stored

            // ---- continuity, src/fluxes.cpp:87-121 ----
            double fr = (RW_(r0, R_RU, -1, 0) - RW_(r0, R_RU, 1, 0)) * hx * dx1;
            fr -= (RW_(r0, R_RV, 0, 1) - RW_(r0, R_RV, 0, -1)) * tmpy;
            double dwz;
            if (EDGE && k == 1 && g.top_edge)
                dwz = (4.0 * RW_(rp, R_RW, 0, 0) - fs.xin[R_RW][nc + 2 * PL]) * tmpz;
            else if (EDGE && k == g.npz && g.bot_edge)
                dwz = (fs.xin[R_RW][nc - 2 * PL] - 4.0 * RM_(R_RW)) * tmpz;
            else
                dwz = (RW_(rp, R_RW, 0, 0) - RM_(R_RW)) * tmpz;
            fr -= dwz;
            if constexpr (IDD && !MHD) {
                // ---- density diffusion (ID 1, 2), 3dmhdsub.f:1316-1386: WW1 = RO - ROM(K) ----
                const double rmk = L.rom[k];
                const double w0 = RW_(r0, R_RO, 0, 0) - rmk;
                if (ph.id_dh != 0.0) {
                    const double wxp = RW_(r0, R_RO, 1, 0) - rmk, wxm = RW_(r0, R_RO, -1, 0) - rmk;
                    const double wyp = RW_(r0, R_RO, 0, 1) - rmk, wym = RW_(r0, R_RO, 0, -1) - rmk;
                    const double ww2 = (wxp - wxm) * hx * d2x + d2sum(wxp, w0, wxm) * h2x * dx1 * dx1;  // :1349
                    const double ww3 = (wyp - wym) * tmpy1 + d2sum(wyp, w0, wym) * tmpy2;                // :1358
                    fr = fr + (ww2 + ww3) * (ph.id_dh_ore * L.wwz[k]);                                   // :1366
                }
                if (ph.id_dv != 0.0) {
                    // rho at k-1, k+1; the domain's ghost planes hold their mirror planes (:1318, :1321)
                    const double ro_m = fs.xin[R_RO][nc - PL], ro_p = RW_(rp, R_RO, 0, 0);
                    const double rzp = (k == g.npz && g.bot_edge) ? ro_m : ro_p;
                    const double rzm = (k == 1 && g.top_edge) ? ro_p : ro_m;
                    const double wzp = rzp - L.rom[k + 1], wzm = rzm - L.rom[k - 1];
                    const double ww2z = (wzp - wzm) * L.tmpz1[k] + d2sum(wzp, w0, wzm) * L.tmpz2[k];     // :1375
                    fr = fr + ww2z * (ph.id_dv_ore * L.wwz[k]);                                          // :1383
                }
            }

            double fu = 0.0, fv = 0.0, fw = 0.0, ft = 0.0;
            double b1 = 0.0, b2f = 0.0, b3 = 0.0;  // B fluxes WW1..WW3 (MHD)
            const double dzk = L.dzzdz[k];
            const double U0 = DV_(d0, D_U, 0, 0), V0 = DV_(d0, D_V, 0, 0), W0 = DV_(d0, D_W, 0, 0);
            const double ri = LEAN ? riq[c] : DV_(d0, D_RI, 0, 0);
            const double Uxp = DV_(d0, D_U, 1, 0), Uxm = DV_(d0, D_U, -1, 0);
            const double Uyp = DV_(d0, D_U, 0, 1), Uym = DV_(d0, D_U, 0, -1);
            const double Uzp = DV_(dp, D_U, 0, 0), Uzm = DV_(dm, D_U, 0, 0);
            const double Vxp = DV_(d0, D_V, 1, 0), Vxm = DV_(d0, D_V, -1, 0);
            const double Vyp = DV_(d0, D_V, 0, 1), Vym = DV_(d0, D_V, 0, -1);
            const double Vzp = DV_(dp, D_V, 0, 0), Vzm = DV_(dm, D_V, 0, 0);
            const double Wxp = DV_(d0, D_W, 1, 0), Wxm = DV_(d0, D_W, -1, 0);
            const double Wyp = DV_(d0, D_W, 0, 1), Wym = DV_(d0, D_W, 0, -1);
            const double Wzp = DV_(dp, D_W, 0, 0), Wzm = DV_(dm, D_W, 0, 0);
            // velocity gradients, the reference's WW1..WW3 / RU..RW temporaries
            const double ux = (Uxp - Uxm) * hx * dx1;  // src/fluxes.cpp:331,416; 3dmhdsub.f:2151
            const double vx = (Vxp - Vxm) * hx * dx1;  // :336; 3dmhdsub.f:2157
            const double wx = (Wxp - Wxm) * hx * dx1;  // :341,505; 3dmhdsub.f:2163
            const double uy = (Uyp - Uym) * hy * dyj;  // :382; 3dmhdsub.f:2181
            const double vy = (Vyp - Vym) * hy * dyj;  // :397; 3dmhdsub.f:2187
            const double wy = (Wyp - Wym) * hy * dyj;  // :476; 3dmhdsub.f:2193
            const double uz = (Uzp - Uzm) * hz * dzk;  // :464; 3dmhdsub.f:2211
            const double vz = (Vzp - Vzm) * hz * dzk;  // :469; 3dmhdsub.f:2217
            const double wz = (Wzp - Wzm) * hz * dzk;  // :423; 3dmhdsub.f:2223

            if (!EDGE || FULLTOP) {
                const double tmpz1 = L.tmpz1[k], tmpz2 = L.tmpz2[k];
                const double T0 = RW_(r0, R_TT, 0, 0);

                // ---- buoyancy and pressure, src/fluxes.cpp:126-152 ----
                fw = ph.grav * RW_(r0, R_RO, 0, 0);
                fw -= (PP_ - PM_) * tmpz;
                fv = (P0_(0, -1) - P0_(0, 1)) * tmpy;
                fu = (P0_(-1, 0) - P0_(1, 0)) * hx * dx1;

                // ---- momentum advection, src/fluxes.cpp:171-224 ----
                fu -= (RW_(r0, R_RU, 1, 0) * Uxp - RW_(r0, R_RU, -1, 0) * Uxm) * hx * dx1;
                fu -= (RW_(r0, R_RU, 0, 1) * Vyp - RW_(r0, R_RU, 0, -1) * Vym) * tmpy;
                fu -= (RW_(rp, R_RU, 0, 0) * Wzp - RM_(R_RU) * Wzm) * tmpz;
                fv -= (RW_(r0, R_RV, 1, 0) * Uxp - RW_(r0, R_RV, -1, 0) * Uxm) * hx * dx1;
                fv -= (RW_(r0, R_RV, 0, 1) * Vyp - RW_(r0, R_RV, 0, -1) * Vym) * tmpy;
                fv -= (RW_(rp, R_RV, 0, 0) * Wzp - RM_(R_RV) * Wzm) * tmpz;
                fw -= (RW_(r0, R_RW, 1, 0) * Uxp - RW_(r0, R_RW, -1, 0) * Uxm) * hx * dx1;
                fw -= (RW_(r0, R_RW, 0, 1) * Vyp - RW_(r0, R_RW, 0, -1) * Vym) * tmpy;
                fw -= (RW_(rp, R_RW, 0, 0) * Wzp - RM_(R_RW) * Wzm) * tmpz;

                // ---- energy advection, src/fluxes.cpp:229-243 ----
                const double Txp = RW_(r0, R_TT, 1, 0), Txm = RW_(r0, R_TT, -1, 0);
                const double Typ = RW_(r0, R_TT, 0, 1), Tym = RW_(r0, R_TT, 0, -1);
                const double Tzp = RW_(rp, R_TT, 0, 0), Tzm = RM_(R_TT);
                ft = -1.0 * U0 * (Txp - Txm) * hx * dx1;
                ft -= V0 * (Typ - Tym) * tmpy;
                ft -= W0 * (Tzp - Tzm) * tmpz;

                // ---- thermal conduction, src/fluxes.cpp:246-276 ----
                const double td = ph.tdiff;
                if (KC) {  // rkapa == 1, dkapa == 0: x*1 == x, ft + (+-0) == ft
                    ft += ((Txp - Txm) * hx * d2x + d2sum(Txp, T0, Txm) * h2x * dx1 * dx1) * ri * td;
                    ft += ((Typ - Tym) * tmpy1 + d2sum(Typ, T0, Tym) * tmpy2) * ri * td;
                    ft += ((Tzp - Tzm) * tmpz1 + d2sum(Tzp, T0, Tzm) * tmpz2) * ri * td;
                } else {
                    const double rk = L.rkapa[k], dk = L.dkapa[k];
                    ft += ((Txp - Txm) * hx * d2x + d2sum(Txp, T0, Txm) * h2x * dx1 * dx1) * ri * td * rk;
                    ft += ((Typ - Tym) * tmpy1 + d2sum(Typ, T0, Tym) * tmpy2) * ri * td * rk;
                    ft += ((Tzp - Tzm) * tmpz1 + d2sum(Tzp, T0, Tzm) * tmpz2) * ri * td * rk;
                    ft += (Tzp - Tzm) * hz * dzk * ri * td * dk;
                }

                // ---- embedded heat loss (itcon 2), 3dmhdsub.f:1799-1821: RO holds 1/rho there ----
                if (ph.heat_on) {
                    double q = ph.heat_pre * ri * L.heat_x[ia];
                    if (!ph.hh_one) q = q / ph.hh;
                    q = q * L.heat_y[ja];
                    if (!ph.hh_one) q = q / ph.hh;
                    q = q * L.heat_z[k];
                    if (!ph.hh_one) q = q / ph.hh;
                    ft = ft - q;
                }

                // ---- viscous momentum, src/fluxes.cpp:281-320 ----
                const double ore = ph.ore, c43 = ph.c43;
                fu += ore * (c43 * ((Uxp - Uxm) * hx * d2x + d2sum(Uxp, U0, Uxm) * h2x * dx1 * dx1) +
                             (Uyp - Uym) * tmpy1 + d2sum(Uyp, U0, Uym) * tmpy2 +
                             (Uzp - Uzm) * tmpz1 + d2sum(Uzp, U0, Uzm) * tmpz2);
                fv += ore * (((Vxp - Vxm) * hx * d2x + d2sum(Vxp, V0, Vxm) * h2x * dx1 * dx1) +
                             c43 * ((Vyp - Vym) * tmpy1 + d2sum(Vyp, V0, Vym) * tmpy2) +
                             (Vzp - Vzm) * tmpz1 + d2sum(Vzp, V0, Vzm) * tmpz2);
                fw += ore * (((Wxp - Wxm) * hx * d2x + d2sum(Wxp, W0, Wxm) * h2x * dx1 * dx1) +
                             (Wyp - Wym) * tmpy1 + d2sum(Wyp, W0, Wym) * tmpy2 +
                             c43 * ((Wzp - Wzm) * tmpz1 + d2sum(Wzp, W0, Wzm) * tmpz2));

                // ---- viscous heating, p dV and cross terms, src/fluxes.cpp:327-514 ----
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
                if (MHD && ph.lrot) {  // hydro: added before the stage update
                    fu += ph.omz * RW_(r0, R_RV, 0, 0);
                    fv += -ph.omz * RW_(r0, R_RU, 0, 0) + ph.omx * RW_(r0, R_RW, 0, 0);
                    fw += -ph.omx * RW_(r0, R_RV, 0, 0);
                }
            }

            if (MHD) {
                // ---- magnetic terms, golden/fortran/3dmhdsub.f:2146-2650 (LMAG branch) ----
                // At k = 1 / npz the momenta, T and Bz are rewritten by BCON afterwards; the
                // Lorentz/ohmic contributions there are computed and discarded like the rest.
                const double h2y = ph.h2y, h2z = ph.h2z, d2y = L.d2yydy2[ja], d2z = L.d2zzdz2[k];
                const double ob = ph.obeta, orm = ph.orm, tmag = ph.tmag;
                const double BX0 = RW_(r0, R_BX, 0, 0), BY0 = RW_(r0, R_BY, 0, 0), BZ0 = RW_(r0, R_BZ, 0, 0);
                const double BXxp = RW_(r0, R_BX, 1, 0), BXxm = RW_(r0, R_BX, -1, 0);
                const double BXyp = RW_(r0, R_BX, 0, 1), BXym = RW_(r0, R_BX, 0, -1);
                const double BXzp = RW_(rp, R_BX, 0, 0), BXzm = RW_(rm, R_BX, 0, 0);
                const double BYxp = RW_(r0, R_BY, 1, 0), BYxm = RW_(r0, R_BY, -1, 0);
                const double BYyp = RW_(r0, R_BY, 0, 1), BYym = RW_(r0, R_BY, 0, -1);
                const double BYzp = RW_(rp, R_BY, 0, 0), BYzm = RW_(rm, R_BY, 0, 0);
                const double BZxp = RW_(r0, R_BZ, 1, 0), BZxm = RW_(r0, R_BZ, -1, 0);
                const double BZyp = RW_(r0, R_BZ, 0, 1), BZym = RW_(r0, R_BZ, 0, -1);
                const double BZzp = RW_(rp, R_BZ, 0, 0), BZzm = RW_(rm, R_BZ, 0, 0);
                // dW/dz with the one-sided forms at the top and bottom planes (2245-2259)
                double wzb = wz;
                if (EDGE && k == 1 && g.top_edge) {
                    const int n2 = nc + 2 * PL;
                    const double w2 = fs.xin[R_RW][n2] * __drcp_rn(fs.xin[R_RO][n2]);
                    wzb = (4.0 * Wzp - w2) * hz * dzk;
                } else if (EDGE && k == g.npz && g.bot_edge) {
                    const int n2 = nc - 2 * PL;
                    const double w2 = fs.xin[R_RW][n2] * __drcp_rn(fs.xin[R_RO][n2]);
                    wzb = (w2 - 4.0 * Wzm) * hz * dzk;
                }
                b2f = BX0 * vx - BY0 * ux;                 // 1030
                b3 = BX0 * wx - BZ0 * ux;                  // 1040
                b1 = BY0 * uy - BX0 * vy;                  // 1080
                b3 = b3 + BY0 * wy - BZ0 * vy;             // 1090
                b1 = b1 + BZ0 * uz - BX0 * wzb;            // 1130
                b2f = b2f + BZ0 * vz - BY0 * wzb;          // 1140
                const double bxx = (BXxp - BXxm) * hx * dx1;   // 1150
                const double byx = (BYxp - BYxm) * hx * dx1;   // 1160
                const double bzx = (BZxp - BZxm) * hx * dx1;   // 1170
                const double bxy = (BXyp - BXym) * hy * dyj;   // 1180
                fu = fu + ob * BY0 * (bxy - byx) - ob * BZ0 * bzx;  // 1190
                fv = fv + ob * BX0 * (byx - bxy);                   // 1200
                fw = fw + ob * BX0 * bzx;                           // 1210
                ft = ft + (bxy * bxy + byx * byx + bzx * bzx - 2.0 * byx * bxy) * ri * tmag;  // 1220
                b1 = b1 - U0 * bxx - V0 * bxy;             // 1230
                b2f = b2f - U0 * byx;                      // 1240
                b3 = b3 - U0 * bzx;                        // 1250
                const double d2bxx = (BXxp - BXxm) * hx * d2x + d2sum(BXxp, BX0, BXxm) * h2x * dx1 * dx1;  // 1260
                const double d2byx = (BYxp - BYxm) * hx * d2x + d2sum(BYxp, BY0, BYxm) * h2x * dx1 * dx1;  // 1265
                const double d2bxy = (BXyp - BXym) * hy * d2y + d2sum(BXyp, BX0, BXym) * h2y * dyj * dyj;  // 1270
                b1 = b1 + orm * (d2bxx + d2bxy);           // 1280
                b2f = b2f + orm * d2byx;                   // 1290
                const double d2bzx = (BZxp - BZxm) * hx * d2x + d2sum(BZxp, BZ0, BZxm) * h2x * dx1 * dx1;  // 1300
                b3 = b3 + orm * d2bzx;                     // 1310
                const double bxz = (BXzp - BXzm) * hz * dzk;   // 1320
                const double byy = (BYyp - BYym) * hy * dyj;   // 1330
                fu = fu + ob * BZ0 * bxz;                  // 1340
                fw = fw - ob * BX0 * bxz;                  // 1350
                ft = ft + (bxz * bxz - 2.0 * bxz * bzx) * ri * tmag;  // 1360
                b1 = b1 - W0 * bxz;                        // 1370
                b2f = b2f - V0 * byy;                      // 1380
                double d2bxz, d2byz;
                if (EDGE && k == 1 && g.top_edge) {  // 1391, 1511
                    const double bx2 = fs.xin[R_BX][nc + 2 * PL], bx3 = fs.xin[R_BX][nc + 3 * PL];
                    const double by2 = fs.xin[R_BY][nc + 2 * PL], by3 = fs.xin[R_BY][nc + 3 * PL];
                    d2bxz = (-3.0 * BX0 + 4.0 * BXzp - bx2) * hz * d2z +
                            (2.0 * BX0 - 5.0 * BXzp + 4.0 * bx2 - bx3) * h2z * dzk * dzk;
                    d2byz = (-3.0 * BY0 + 4.0 * BYzp - by2) * hz * d2z +
                            (2.0 * BY0 - 5.0 * BYzp + 4.0 * by2 - by3) * h2z * dzk * dzk;
                } else if (EDGE && k == g.npz && g.bot_edge) {  // 1392, 1513
                    const double bx2 = fs.xin[R_BX][nc - 2 * PL], bx3 = fs.xin[R_BX][nc - 3 * PL];
                    const double by2 = fs.xin[R_BY][nc - 2 * PL], by3 = fs.xin[R_BY][nc - 3 * PL];
                    d2bxz = (3.0 * BX0 - 4.0 * BXzm + bx2) * hz * d2z +
                            (2.0 * BX0 - 5.0 * BXzm + 4.0 * bx2 - bx3) * h2z * dzk * dzk;
                    d2byz = (3.0 * BY0 - 4.0 * BYzm + by2) * hz * d2z +
                            (2.0 * BY0 - 5.0 * BYzm + 4.0 * by2 - by3) * h2z * dzk * dzk;
                } else {  // 1390, 1510
                    d2bxz = (BXzp - BXzm) * hz * d2z + d2sum(BXzp, BX0, BXzm) * h2z * dzk * dzk;
                    d2byz = (BYzp - BYzm) * hz * d2z + d2sum(BYzp, BY0, BYzm) * h2z * dzk * dzk;
                }
                const double d2byy = (BYyp - BYym) * hy * d2y + d2sum(BYyp, BY0, BYym) * h2y * dyj * dyj;  // 1400
                b1 = b1 + orm * d2bxz;                     // 1410
                b2f = b2f + orm * d2byy;                   // 1420
                const double byz = (BYzp - BYzm) * hz * dzk;   // 1430
                const double bzy = (BZyp - BZym) * hy * dyj;   // 1440
                const double cy = byz - bzy;               // 1450
                fv = fv + ob * BZ0 * cy;                   // 1460
                fw = fw - ob * BY0 * cy;                   // 1470
                ft = ft + (byz * byz + bzy * bzy - 2.0 * byz * bzy) * ri * tmag;  // 1480
                b2f = b2f - W0 * byz;                      // 1490
                b3 = b3 - V0 * bzy;                        // 1500
                const double d2bzy = (BZyp - BZym) * hy * d2y + d2sum(BZyp, BZ0, BZym) * h2y * dyj * dyj;  // 1520
                b2f = b2f + orm * d2byz;                   // 1530
                b3 = b3 + orm * d2bzy;                     // 1540
                const double bzz = (BZzp - BZzm) * hz * dzk;   // 1550
                b3 = b3 - W0 * bzz;                        // 1560
                const double d2bzz = (BZzp - BZzm) * hz * d2z + d2sum(BZzp, BZ0, BZzm) * h2z * dzk * dzk;  // 1570
                b3 = b3 + orm * d2bzz;                     // 1580
                if (EDGE) {  // the hydro fluxes there are rewritten by BCON: keep them finite
                    fu = fv = fw = ft = 0.0;
                }
            }
            Fc[c][0] = fu;
            Fc[c][1] = fv;
            Fc[c][2] = fw;
            Fc[c][3] = fr;
            Fc[c][4] = ft;
            if constexpr (MHD) {
                Fc[c][5] = b1;
                Fc[c][6] = b2f;
                Fc[c][7] = b3;
            }
          }
        };
        if (!edge) {
            rhs(EdgeTag<false>{});
        } else {
            if constexpr ((TF || IDD) && !MHD) {
                if (k == 1 && g.top_edge && (TF || ph.top_free)) rhs(EdgeTag<true, true>{});
                else rhs(EdgeTag<true>{});
            } else {
                rhs(EdgeTag<true>{});
            }
        }
        if constexpr (LEAN) {
            // hydro: this plane's accumulators (prefetched into L2 a plane earlier), loaded after
            // the fluxes; the compiler barrier keeps the loads from being hoisted into them
            asm volatile("" ::: "memory");
#pragma unroll
            for (int c = 0; c < CPT; ++c) {
#pragma unroll
                for (int f = 0; f < NF; ++f) zq[c][f] = 0.0;
                if (STAGE > 0 && actv[c]) {
#pragma unroll
                    for (int f = 0; f < NF; ++f) zq[c][f] = fs.z[f][k * PL + colv[c]];
                }
            }
        }
#pragma unroll
        for (int c = 0; c < CPT; ++c) {
          if (actv[c]) {
            // ---- stage update, src/step.cpp:53-110 (B: 3dmhdsub.f:957-973, 1059-1075, 1161-1177) ----
            const int j = jr + c;
            const int s0 = (ty * CPT + c + 1) * SX + (tx + 1);
            const int nc = k * PL + colv[c];
            double* F = Fc[c];
            if (!MHD && !edge && ph.lrot) {  // rotation, src/fluxes.cpp:519-533 (the last terms)
                F[0] += ph.omz * RW_(r0, R_RV, 0, 0);
                F[1] += -ph.omz * RW_(r0, R_RU, 0, 0) + ph.omx * RW_(r0, R_RW, 0, 0);
                F[2] += -ph.omx * RW_(r0, R_RV, 0, 0);
            }
            const int gdy = (j == 1) ? g.npy * PX : ((j == g.npy) ? -g.npy * PX : 0);
            const bool ghost = gdx != 0 || gdy != 0;
            double xn[NF];
#pragma unroll
            for (int f = 0; f < NF; ++f) {
                const double zv = (STAGE == 0) ? RW_(r0, f, 0, 0) : zq[c][f];
                xn[f] = zv + cg * F[f];
                fs.xout[f][nc] = xn[f];
                if (STAGE < 2) fs.z[f][nc] = xn[f] + cz * F[f];
                if constexpr (EMIT) fs.f[f][nc] = F[f];  // the adjoint's recompute keeps F
            }
            if (ghost) {  // periodic images (src/communicate.cpp:108-168), edge threads only
#pragma unroll
                for (int f = 0; f < NF; ++f) {
                    if (gdx) fs.xout[f][nc + gdx] = xn[f];
                    if (gdy) fs.xout[f][nc + gdy] = xn[f];
                    if (gdx && gdy) fs.xout[f][nc + gdx + gdy] = xn[f];
                }
            }
            if (STAGE == 2 && !edge) {
                const double dd = (L.ddz[k] < dxyv[c]) ? L.ddz[k] : dxyv[c];  // min_of3(ddx, ddy, ddz)
                double b2sum = 0.0;
                if constexpr (MHD) b2sum = xn[5] * xn[5] + xn[6] * xn[6] + xn[7] * xn[7];
                if (s_filter) {
                    fold_dt_filtered<KC, MHD>(ph, xn[0], xn[1], xn[2], xn[3], xn[4], b2sum, dd,
                                              L.rkapa[k], s_thr[0], s_thr[1], m1, m2, m3, m4, mu);
                } else {
                    double w1, w2, w3, w4, um;
                    dt_terms<KC>(ph, xn[0], xn[1], xn[2], xn[3], xn[4], b2sum, dd, L.rkapa[k], w1,
                                 w2, w3, w4, um);
                    m1 = fold_min(m1, w1);
                    m2 = fold_min(m2, w2);
                    m3 = fold_min(m3, w3);
                    m4 = fold_min(m4, w4);
                    mu = fold_max(mu, um);
                }
            }
          }
        }
        if constexpr (LEAN) {  // this plane's own-cell values become the next plane's k-1 values
#pragma unroll
            for (int c = 0; c < CPT; ++c) {
                const int s0 = own0 + c * SX;
#pragma unroll
                for (int f = 0; f < 5; ++f) cm[c][f] = RW_(r0, f, 0, 0);
                cm[c][R_RO] = RW_(r0, R_RO, 0, 0) * RW_(r0, R_TT, 0, 0);  // the plane's own P
            }
        }
#undef RM_
#undef P0_
#undef PP_
#undef PM_
#undef RW_
#undef DV_
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

template <int STAGE, bool KC, bool MHD, bool EMIT, int TYV, bool TF, bool IDD>
static void launch_one(dim3 grid, const StageMaps& maps, const Geometry& g, const Physics& ph,
                       const Lines& L, const FieldSet& fs, Scalars* sc, int kchunk, cudaStream_t st) {
    static bool configured = false;
    constexpr size_t smem = Shape<MHD, TYV>::smem;
    if (!configured) {
        cudaFuncSetAttribute(stage_fp64<STAGE, KC, MHD, EMIT, TYV, TF, IDD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
        // all of the unified L1 as shared memory, so that the resident CTAs fit
        cudaFuncSetAttribute(stage_fp64<STAGE, KC, MHD, EMIT, TYV, TF, IDD>,
                             cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        configured = true;
    }
    const dim3 block(TX, TYV / Cells<MHD, STAGE, TYV>::cpt, 1);
    stage_fp64<STAGE, KC, MHD, EMIT, TYV, TF, IDD><<<grid, block, smem, st>>>(maps, g, ph, L, fs, sc, kchunk);
}

template <bool MHD, bool EMIT, int TYV, bool TF = false, bool IDD = false>
static void launch_stage(int stage, const StageMaps& maps, const Geometry& g, const Physics& ph,
                         const Lines& L, const FieldSet& fs, Scalars* sc, int kchunk, cudaStream_t st) {
    const dim3 grid((g.npx + TX - 1) / TX, (g.npy + TYV - 1) / TYV, (g.npz + kchunk - 1) / kchunk);
    const bool kc = ph.kappa_const != 0;
    if (stage == 0) kc ? launch_one<0, true, MHD, EMIT, TYV, TF, IDD>(grid, maps, g, ph, L, fs, sc, kchunk, st)
                       : launch_one<0, false, MHD, EMIT, TYV, TF, IDD>(grid, maps, g, ph, L, fs, sc, kchunk, st);
    else if (stage == 1) kc ? launch_one<1, true, MHD, EMIT, TYV, TF, IDD>(grid, maps, g, ph, L, fs, sc, kchunk, st)
                            : launch_one<1, false, MHD, EMIT, TYV, TF, IDD>(grid, maps, g, ph, L, fs, sc, kchunk, st);
    else kc ? launch_one<2, true, MHD, EMIT, TYV, TF, IDD>(grid, maps, g, ph, L, fs, sc, kchunk, st)
            : launch_one<2, false, MHD, EMIT, TYV, TF, IDD>(grid, maps, g, ph, L, fs, sc, kchunk, st);
}

template <bool EMIT>
static void launch_any(int stage, const StageMaps& maps, const Geometry& g, const Physics& ph,
                       const Lines& L, const FieldSet& fs, Scalars* sc, int kchunk, cudaStream_t st) {
    if constexpr (!EMIT) {  // ID, itcon 3 (hydro; the adjoint's EMIT recompute refuses them)
        if (!ph.lmag && ph.id_mode) {
            launch_stage<false, false, R3D_STAGE_TY, false, true>(stage, maps, g, ph, L, fs, sc, kchunk, st);
            return;
        }
        if (!ph.lmag && ph.top_free) {
            launch_stage<false, false, R3D_STAGE_TY, true>(stage, maps, g, ph, L, fs, sc, kchunk, st);
            return;
        }
    }
    if (!ph.lmag) launch_stage<false, EMIT, R3D_STAGE_TY>(stage, maps, g, ph, L, fs, sc, kchunk, st);
    else if (g.tile_rows == 6) launch_stage<true, EMIT, 6>(stage, maps, g, ph, L, fs, sc, kchunk, st);
    else launch_stage<true, EMIT, 8>(stage, maps, g, ph, L, fs, sc, kchunk, st);
}

cudaError_t launch_stage_fp64(int stage, const StageMaps& maps, const Geometry& g,
                              const Physics& ph, const Lines& L, const FieldSet& fs, Scalars* sc,
                              int kchunk, cudaStream_t st, bool emit_rhs) {
    if (ph.lmag && g.tile_rows != 6 && g.tile_rows != 8) return cudaErrorInvalidValue;
    if (!ph.lmag && g.tile_rows != R3D_STAGE_TY) return cudaErrorInvalidValue;
    if (emit_rhs) launch_any<true>(stage, maps, g, ph, L, fs, sc, kchunk, st);
    else launch_any<false>(stage, maps, g, ph, L, fs, sc, kchunk, st);
    return cudaGetLastError();
}

}  // namespace r3dk
