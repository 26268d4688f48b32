// bcon.cu - BCON, ghost images, time-step limits and scalar bookkeeping kernels.
//
// BCON (src/bcon.cpp:12-141) rewrites planes 1 and npz after every stage; after the third stage
// it also evaluates the time-step limits of those two planes (the stage kernel covers the
// others).  dt_full evaluates the limits of a whole state (after an upload or a partial step).
// step_begin/step_end keep dt, umach, nit, timc, timt on the device (src/step.cpp:133-256).
#include <cuda_runtime.h>

#include "r3d_kernels.h"
#include "stage_common.cuh"

namespace r3dk {

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
        // top, k = 1 (src/bcon.cpp:27-98); a z slab that does not hold the domain's top
        // plane has a neighbour's ghost plane there instead
        if (g.top_edge) {
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
                case 5: t = tt[n]; break;  // itcon 3: the stage's value stands
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
        if (g.bot_edge) {
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

// ---------------------------------------------------------------------------------------
// Horizontal mean of rho per plane for the density diffusion (ID 1, 2): HORIZONTAL_MEAN of the
// Fortran (3dmhdsub.f:3177-3186, the uniform grid it requires, one rank in y): the plane's
// interior values added in loop order (j outer, i inner) and divided by FLOAT(NPX*NPY).  One
// CTA per plane: its other warps stage the plane in chunks of kMeanChunk values (in that
// order, coalesced, double-buffered in shared memory) while thread 0 adds them one by one, so
// the order is exactly the Fortran's.  The domain's ghost planes are first loaded with their
// mirror planes (3dmhdsub.f:1318, 1321), so their means are those of planes 2 and npz-1.
// ---------------------------------------------------------------------------------------
constexpr int kMeanChunk = 2048, kMeanThreads = 256;

__global__ void __launch_bounds__(kMeanThreads) plane_mean_kernel(Geometry g, const double* ro, double* rom,
                                                                   double* wwz, int id_mode) {
    __shared__ double buf[2][kMeanChunk];
    const int k = blockIdx.x;  // local plane 0 .. npz+1
    int src = k;
    if (k == 0 && g.top_edge) src = 2;
    if (k == g.npz + 1 && g.bot_edge) src = g.npz - 1;
    const double* p = ro + (int64_t)src * g.plane;
    const int64_t nval = (int64_t)g.npx * g.npy;
    const int nchunk = (int)((nval + kMeanChunk - 1) / kMeanChunk);
    // value t of the plane in (j, i) order: row 1 + t / npx, column 1 + t % npx
    auto load = [&](int c, double* b) {
        if (threadIdx.x < 32) return;  // warp 0 adds
        const int64_t t0 = (int64_t)c * kMeanChunk;
        for (int u = threadIdx.x - 32; u < kMeanChunk; u += kMeanThreads - 32) {
            const int64_t t = t0 + u;
            if (t < nval) b[u] = p[(1 + t / g.npx) * g.pitch + 1 + t % g.npx];
        }
    };
    load(0, buf[0]);
    __syncthreads();
    double sum = 0.0;
    for (int c = 0; c < nchunk; ++c) {
        if (c + 1 < nchunk) load(c + 1, buf[(c + 1) & 1]);
        if (threadIdx.x == 0) {
            const double* b = buf[c & 1];
            const int n = (int)min((int64_t)kMeanChunk, nval - (int64_t)c * kMeanChunk);
            for (int u = 0; u < n; ++u) sum = sum + b[u];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double m = sum / (double)(float)(g.npx * g.npy);
        rom[k] = m;
        if (id_mode == 1) wwz[k] = 1.0 / m;  // WWZ = 1.0E00/ROM (3dmhdsub.f:1338)
    }
}

cudaError_t launch_plane_mean(const Geometry& g, const double* ro, double* rom, double* wwz, int id_mode,
                              cudaStream_t st) {
    plane_mean_kernel<<<g.npz + 2, kMeanThreads, 0, st>>>(g, ro, rom, wwz, id_mode);
    return cudaGetLastError();
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
                                                      FieldSet fs, Scalars* sc, int only_refold) {
    __shared__ double red[5 * 8];
    if (only_refold && *(volatile int*)&sc->refold == 0) return;  // uniform over the grid
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
                           const FieldSet& fs, Scalars* sc, cudaStream_t st, int only_refold) {
    dim3 block(32, 8, 1);
    // the conditional form (after a filtered third stage) is a no-op in almost every step: a
    // shallow grid keeps its cost to a few microseconds
    dim3 grid((g.npx + 31) / 32, (g.npy + 7) / 8, (unsigned)min(g.npz, only_refold ? 2 : 64));
    dt_full_kernel<<<grid, block, 0, st>>>(g, ph, L, fs, sc, only_refold);
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
    const double u = order_value(sc->umax);
    sc->umach = sqrt(u);
    // thresholds of this step's filtered fold: the previous limits widened by the margin (a
    // margin < 0 forces the re-evaluation path; thr_on == 0 leaves only the exact running bounds);
    // a slab takes its own limits, so that its check at step_end makes its own fold exact
    const double tw = sc->thr_local ? order_value(sc->wloc[0]) : w0;
    const double tu = sc->thr_local ? order_value(sc->uloc) : u;
    sc->thr_w1 = sc->thr_on ? tw * (1.0 + sc->thr_margin) : 1e308;
    sc->thr_um = sc->thr_on ? tu * (1.0 - sc->thr_margin) : 0.0;
    sc->wmin[0] = sc->wmin[1] = sc->wmin[2] = sc->wmin[3] = order_key(1e300);
    sc->umax = order_key(0.0);
}

// check != 0 (after a full step on a handle with the threshold filter): the skipped cells have
// ww1 > thr_w1 and a Mach term < thr_um, so the folded limits are exact iff the minimum found
// is <= thr_w1 and the maximum >= thr_um; otherwise clear them and request the full evaluation
// (dt_full_kernel with only_refold).
__global__ void step_end_kernel(Scalars* sc, int check) {
    sc->nit += 1;
    sc->timc += sc->dt;
    sc->timt = sc->timi + sc->timc;
    int refold = 0;
    if (check && sc->thr_on) {
        refold = !(order_value(sc->wmin[0]) <= sc->thr_w1) || !(order_value(sc->umax) >= sc->thr_um);
        if (refold) {
            sc->refolds += 1;
            sc->wmin[0] = sc->wmin[1] = sc->wmin[2] = sc->wmin[3] = order_key(1e300);
            sc->umax = order_key(0.0);
        }
    }
    sc->refold = refold;
}

__global__ void save_local_limits_kernel(Scalars* sc) {
    for (int q = 0; q < 4; ++q) sc->wloc[q] = sc->wmin[q];
    sc->uloc = sc->umax;
}

__global__ void reset_reduction_kernel(Scalars* sc) {
    sc->wmin[0] = sc->wmin[1] = sc->wmin[2] = sc->wmin[3] = order_key(1e300);
    sc->umax = order_key(0.0);
}

cudaError_t launch_step_begin(const Physics& ph, Scalars* sc, cudaStream_t st) {
    step_begin_kernel<<<1, 1, 0, st>>>(ph, sc);
    return cudaGetLastError();
}
cudaError_t launch_step_end(Scalars* sc, cudaStream_t st, int check) {
    step_end_kernel<<<1, 1, 0, st>>>(sc, check);
    return cudaGetLastError();
}
cudaError_t launch_save_local_limits(Scalars* sc, cudaStream_t st) {
    save_local_limits_kernel<<<1, 1, 0, st>>>(sc);
    return cudaGetLastError();
}
cudaError_t launch_reset_reduction(Scalars* sc, cudaStream_t st) {
    reset_reduction_kernel<<<1, 1, 0, st>>>(sc);
    return cudaGetLastError();
}

}  // namespace r3dk
