// bcon_fp32.cu - BCON, time-step limits and totals for the FP32-bulk state.
//
// The state is stored as FP32 momenta and FP32 deviations rho' = rho - R(k), T' = T - T0(k);
// these kernels rebuild full values in FP64 (R, T0 from the static polytrope), apply the
// reference formulas in FP64 (src/bcon.cpp:12-141, src/step.cpp:122-229) and store the result
// back as FP32 deviations.
#include <cuda_runtime.h>

#include "r3d_kernels.h"
#include "stage_common.cuh"

namespace r3dk {

__global__ void __launch_bounds__(256) bcon_fp32_kernel(Geometry g, Physics ph, Lines L, Boundary b,
                                                        Background bg, FieldSet32 fs, Scalars* sc,
                                                        int with_dt) {
    __shared__ double red[5 * 8];
    const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
    const bool active = (i <= g.npx) && (j <= g.npy);
    double m1 = 1e300, m2 = 1e300, m3 = 1e300, m4 = 1e300, mu = 0.0;
    if (active) {
        float* ru = fs.xout[0];
        float* rv = fs.xout[1];
        float* rw = fs.xout[2];
        float* ro = fs.xout[3];
        float* tt = fs.xout[4];
        const double c13 = ph.c13, c23 = ph.c23, c43 = ph.c43;
        const int64_t P = g.plane, row = (int64_t)j * g.pitch + i;
        for (int side = 0; side < 2; ++side) {
            if (side == 0 ? !g.top_edge : !g.bot_edge) continue;  // slab interior face
            const int k = side == 0 ? 1 : g.npz;
            const int dk = side == 0 ? 1 : -1;
            const int64_t n = (int64_t)k * P + row, n1 = n + dk * P, n2 = n + 2 * dk * P;
            const double ro0 = bg.r[k] + (double)ro[n];
            const double ro1 = bg.r[k + dk] + (double)ro[n1];
            const double ro2 = bg.r[k + 2 * dk] + (double)ro[n2];
            const double u = ro0 * (c43 * (double)ru[n1] / ro1 - c13 * (double)ru[n2] / ro2);
            const double v = ro0 * (c43 * (double)rv[n1] / ro1 - c13 * (double)rv[n2] / ro2);
            const double t1 = bg.t[k + dk] + (double)tt[n1], t2 = bg.t[k + 2 * dk] + (double)tt[n2];
            double t;
            if (side == 0) {
                switch (b.top_mode) {
                    case 0: t = 1.0; break;
                    case 1: t = c43 * t1 - c13 * t2 - c23 * b.dz_top * b.theta; break;
                    case 2: t = 1.0 - (1.0 - b.tpr) * L.plume_x[i] / b.hh * L.plume_y[j] / b.hh; break;
                    case 3:
                        t = c43 * t1 - c13 * t2 -
                            c23 * b.dz_top * (b.theta - (b.theta - b.tpr) * L.plume_x[i] / b.hh * L.plume_y[j] / b.hh);
                        break;
                    default: t = (i <= b.half_nx) ? 1.0 - b.tp : 1.0; break;
                }
            } else {
                t = (b.bottom_mode == 0) ? b.tb : c43 * t1 - c13 * t2 + c23 * b.dz_bot * b.theta / L.rkapa[k];
            }
            const int64_t base = (int64_t)k * P;
            put_periodic(ru, base, g, i, j, (float)u);
            put_periodic(rv, base, g, i, j, (float)v);
            put_periodic(rw, base, g, i, j, 0.0f);
            put_periodic(tt, base, g, i, j, (float)(t - bg.t[k]));
            if (with_dt) {
                const double dd = min_of3(L.ddx[i], L.ddy[j], L.ddz[k]);
                double w1, w2, w3, w4, um;
                dt_terms<false>(ph, (double)(float)u, (double)(float)v, 0.0, ro0,
                                bg.t[k] + (double)(float)(t - bg.t[k]), 0.0, dd, L.rkapa[k], w1, w2, w3, w4, um);
                m1 = fold_min(m1, w1);
                m2 = fold_min(m2, w2);
                m3 = fold_min(m3, w3);
                mu = fold_max(mu, um);
            }
        }
    }
    if (with_dt) reduce_dt(red, m1, m2, m3, m4, mu, sc);
}

__global__ void __launch_bounds__(256) dt_full_fp32_kernel(Geometry g, Physics ph, Lines L,
                                                           Background bg, FieldSet32 fs, Scalars* sc,
                                                           int only_refold) {
    __shared__ double red[5 * 8];
    if (only_refold && *(volatile int*)&sc->refold == 0) return;  // uniform over the grid
    const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
    double m1 = 1e300, m2 = 1e300, m3 = 1e300, m4 = 1e300, mu = 0.0;
    if (i <= g.npx && j <= g.npy) {
        const double dxy = (L.ddy[j] < L.ddx[i]) ? L.ddy[j] : L.ddx[i];
        for (int k = 1 + blockIdx.z; k <= g.npz; k += gridDim.z) {
            const int64_t n = (int64_t)k * g.plane + (int64_t)j * g.pitch + i;
            const double dd = (L.ddz[k] < dxy) ? L.ddz[k] : dxy;
            double w1, w2, w3, w4, um;
            dt_terms<false>(ph, fs.xin[0][n], fs.xin[1][n], fs.xin[2][n], bg.r[k] + (double)fs.xin[3][n],
                            bg.t[k] + (double)fs.xin[4][n], 0.0, dd, L.rkapa[k], w1, w2, w3, w4, um);
            m1 = fold_min(m1, w1);
            m2 = fold_min(m2, w2);
            m3 = fold_min(m3, w3);
            mu = fold_max(mu, um);
        }
    }
    reduce_dt(red, m1, m2, m3, m4, mu, sc);
}

__global__ void totals_fp32_kernel(Geometry g, Physics ph, Background bg, FieldSet32 fs, Scalars* sc) {
    const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
    double m = 0.0, e = 0.0;
    if (i <= g.npx && j <= g.npy) {
        for (int k = 1 + blockIdx.z; k <= g.npz; k += gridDim.z) {
            const int64_t n = (int64_t)k * g.plane + (int64_t)j * g.pitch + i;
            const double ru = fs.xin[0][n], rv = fs.xin[1][n], rw = fs.xin[2][n];
            const double ro = bg.r[k] + (double)fs.xin[3][n], tt = bg.t[k] + (double)fs.xin[4][n];
            m += ro;
            e += ro * tt * ph.cv + 0.5 * (ru * ru + rv * rv + rw * rw) / ro;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        m += __shfl_xor_sync(0xffffffffu, m, o);
        e += __shfl_xor_sync(0xffffffffu, e, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&sc->mass, m);
        atomicAdd(&sc->energy, e);
    }
}

cudaError_t launch_bcon_fp32(const Geometry& g, const Physics& ph, const Lines& L, const Boundary& b,
                             const Background& bg, const FieldSet32& fs, Scalars* sc, int with_dt,
                             cudaStream_t st) {
    dim3 block(32, 8, 1), grid((g.npx + 31) / 32, (g.npy + 7) / 8, 1);
    bcon_fp32_kernel<<<grid, block, 0, st>>>(g, ph, L, b, bg, fs, sc, with_dt);
    return cudaGetLastError();
}

cudaError_t launch_dt_full_fp32(const Geometry& g, const Physics& ph, const Lines& L,
                                const Background& bg, const FieldSet32& fs, Scalars* sc, cudaStream_t st,
                                int only_refold) {
    dim3 block(32, 8, 1), grid((g.npx + 31) / 32, (g.npy + 7) / 8, (unsigned)min(g.npz, only_refold ? 2 : 64));
    dt_full_fp32_kernel<<<grid, block, 0, st>>>(g, ph, L, bg, fs, sc, only_refold);
    return cudaGetLastError();
}

cudaError_t launch_totals_fp32(const Geometry& g, const Physics& ph, const Background& bg,
                               const FieldSet32& fs, Scalars* sc, cudaStream_t st) {
    dim3 block(32, 8, 1), grid((g.npx + 31) / 32, (g.npy + 7) / 8, (unsigned)min(g.npz, 64));
    totals_fp32_kernel<<<grid, block, 0, st>>>(g, ph, bg, fs, sc);
    return cudaGetLastError();
}

}  // namespace r3dk
