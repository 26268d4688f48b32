// stage_common.cuh - device helpers shared by the stage, BCON and dt kernels.
#pragma once

#include <cuda_runtime.h>

#include "r3d_device.cuh"

namespace r3dk {

// Per-cell time-step limits of src/step.cpp:125-196 for one cell of the finished state:
// returns ww1 = dd/sqrt(c^2), ww2 (conduction), ww3 (viscosity), vv (resistivity, 1e300 without
// LMAG) and the Mach term ogamma*uu/tt.  b2sum = bx^2+by^2+bz^2 (0 without LMAG).
// KC: rkapa == 1 everywhere, where x/rkapa == x exactly and the division is skipped.
template <bool KC = false>
__device__ __forceinline__ void dt_terms(const Physics& ph, double ru, double rv, double rw,
                                         double ro, double tt, double b2sum, double dd,
                                         double rkap, double& w1, double& w2, double& w3,
                                         double& w4, double& um) {
    const double r = __drcp_rn(ro);  // == 1.0/ro
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
    w2 = KC ? 0.5 * dd * dd * ph.repr * ph.cv * ro : 0.5 * dd * dd * ph.repr * ph.cv * ro / rkap;
    w3 = 0.375 * dd * dd * ph.re * ro;
}

// std::min(acc, v) / std::max(acc, v): a NaN v never replaces acc.
__device__ __forceinline__ double fold_min(double acc, double v);
__device__ __forceinline__ double fold_max(double acc, double v);

// True when x is positive and 2^-30 <= x < 2^31 (one integer compare on the high word): the
// window in which the float estimates below keep their error bound.
__device__ __forceinline__ bool est_window(double x) {
    return (unsigned)__double2hiint(x) - 0x3e100000u < 0x03d00000u;
}

// Fold one cell's time-step limits into running minima m1..m4 and maximum mu.  The cheap limits
// (ww2, ww3, vv: products of the cell's spacing and density) are folded exactly.  The costly
// FP64 ww1 = dd/sqrt(c^2) and Mach term (a reciprocal, two divisions, two square roots) are
// evaluated only for cells that can change m1 or mu: float estimates of both, with relative
// error below 2^-17 (at most thirty float operations on positive quantities, each correctly
// rounded or within 2 ulp, inputs in the est_window range), are compared under a 2^-12 margin
// with b1 = min(m1, t1) and bu = max(mu, tu).  A cell is skipped only when its estimates are
// clearly worse than both bounds; cells outside the window, with a non-finite estimate, or
// while bu <= 2^-40 (where float underflow voids the bound on the Mach term) are evaluated.
// With t1 = +huge and tu = 0 the running values equal those of folding the FP64 values of every
// cell.  With thresholds t1, tu the skipped cells have ww1 > t1 and Mach term < tu, so the
// folded limits over the whole domain are exact whenever the final minimum is <= t1 and the
// final maximum is >= tu (checked by step_end_kernel, which requests a full re-evaluation
// otherwise).  Expressions and operation order of the exact path are those of dt_terms.
template <bool KC, bool MHD>
__device__ __forceinline__ void fold_dt_filtered(const Physics& ph, double ru, double rv,
                                                 double rw, double ro, double tt, double b2sum,
                                                 double dd, double rkap, double t1, double tu,
                                                 double& m1, double& m2, double& m3, double& m4,
                                                 double& mu) {
    m2 = fold_min(m2, KC ? 0.5 * dd * dd * ph.repr * ph.cv * ro                  // src/step.cpp:192-193
                         : 0.5 * dd * dd * ph.repr * ph.cv * ro / rkap);
    m3 = fold_min(m3, 0.375 * dd * dd * ph.re * ro);                            // src/step.cpp:194
    if constexpr (MHD) m4 = fold_min(m4, 0.5 * dd * dd * ph.rm);
    const float rof = (float)ro, ttf = (float)tt;
    const float ruf = (float)ru, rvf = (float)rv, rwf = (float)rw;
    const float rf = __fdividef(1.0f, rof);
    const float uuf = (ruf * ruf + rvf * rvf + rwf * rwf) * rf * rf;
    const float umf = __fdividef(ph.ogamma_f * uuf, ttf);
    const float gtf = ph.gamma_f * ttf;
    float c2f;
    // square roots as x * rsqrt(x) (2 ulp each; 0 for x == 0)
    auto sqrt_est = [](float x) { return x > 0.0f ? x * rsqrtf(x) : 0.0f; };
    if constexpr (MHD) {
        const float b2f = (float)b2sum * ph.obeta_f * rf;
        c2f = uuf + gtf + b2f + 2.0f * sqrt_est(uuf * (gtf + b2f));
    } else {
        c2f = uuf + gtf + 2.0f * sqrt_est(uuf * gtf);
    }
    const float w1f = (float)dd * rsqrtf(c2f);
    const double b1 = (t1 < m1) ? t1 : m1;
    const double bu = (mu < tu) ? tu : mu;
    const bool ok = est_window(ro) && est_window(tt) && est_window(dd);
    const bool skip_um = ok && bu > 0x1p-40 && (double)umf * (1.0 + 1.0 / 4096.0) < bu;
    const bool skip_w1 = ok && (double)w1f * (1.0 - 1.0 / 4096.0) > b1;
    if (skip_um && skip_w1) return;
    double w1, w2, w3, w4, um;
    dt_terms<KC>(ph, ru, rv, rw, ro, tt, MHD ? b2sum : 0.0, dd, rkap, w1, w2, w3, w4, um);
    m1 = fold_min(m1, w1);
    mu = fold_max(mu, um);
}

// std::min(std::min(a, b), c) with the reference's comparison order.
__device__ __forceinline__ double min_of3(double a, double b, double c) {
    const double m = (b < a) ? b : a;
    return (c < m) ? c : m;
}
// std::min(acc, v) / std::max(acc, v): a NaN v never replaces acc.
__device__ __forceinline__ double fold_min(double acc, double v) { return (v < acc) ? v : acc; }
__device__ __forceinline__ double fold_max(double acc, double v) { return (acc < v) ? v : acc; }

// Block-wide fold of the running limits, then one atomic per quantity into the scalars.
// red must hold 5 doubles per warp.  Every thread of the block must call it.
__device__ __forceinline__ void reduce_dt(double* red, double w1, double w2, double w3,
                                          double w4, double um, Scalars* sc) {
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

// Store v at (i,j) of the plane starting at base, and at its periodic ghost images (the
// one-domain form of the periodic exchange, src/communicate.cpp:108-168).
template <class T>
__device__ __forceinline__ void put_periodic(T* f, int64_t base, const Geometry& g, int i, int j,
                                             T v) {
    f[base + (int64_t)j * g.pitch + i] = v;
    const int gi = (i == 1) ? g.npx + 1 : ((i == g.npx) ? 0 : -1);
    const int gj = (j == 1) ? g.npy + 1 : ((j == g.npy) ? 0 : -1);
    if (gi >= 0) f[base + (int64_t)j * g.pitch + gi] = v;
    if (gj >= 0) f[base + (int64_t)gj * g.pitch + i] = v;
    if (gi >= 0 && gj >= 0) f[base + (int64_t)gj * g.pitch + gi] = v;
}

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

}  // namespace r3dk
