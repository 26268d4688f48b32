// r3d_gpu.cu - the C ABI behind include/r3d_gpu.h: device state, upload/download and the
// step sequence.
//
// Replaces GpuSim / gpu_alloc / gpu_upload / gpu_download / gpu_free / step_gpu
// (src/gpu.cpp:185-384, 736-1052).  Differences by design:
//  * the whole global domain lives on one device; the reference's y/z halo exchange becomes
//    the ghost images that the stage and BCON kernels write (no MPI, no NCCL, no staging);
//  * the state is double-buffered (X_a -> X_b) plus one accumulator Z per field, 15 arrays for
//    hydro instead of the reference's 28 (F, UU.., WW1..3 and the rho snapshot are never
//    stored);
//  * dt, umach, nit, timc, timt live on the device; a step is 9 kernel launches (step_begin,
//    3 x (stage, BCON), step_end, the conditional dt_full) with no host round trip (the reference copies three full arrays to the host per step for dt,
//    src/gpu.cpp:790-823).
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <memory>
#include <queue>
#include <string>
#include <vector>

#include "r3d_device.cuh"
#include "r3d_error.hpp"
#include "r3d_gpu.h"
#include "r3d_host.hpp"
#include "r3d_kernels.h"
#include "r3d_gpu_impl.hpp"

using namespace r3db;
using namespace r3dg;
using r3dk::FieldSet;

namespace {

// cuTensorMapEncodeTiled through the runtime's driver entry point (no libcuda link needed).
using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                 const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                 const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                 CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiled encode_fn() {
    static EncodeTiled fn = nullptr;
    if (!fn) {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        cuda_ok(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q),
                "cudaGetDriverEntryPoint(cuTensorMapEncodeTiled)");
        if (!f || q != cudaDriverEntryPointSuccess) throw Error(R3D_ECUDA, "cuTensorMapEncodeTiled unavailable");
        fn = (EncodeTiled)f;
    }
    return fn;
}

}  // namespace

namespace r3dg {

// 3D map over one padded field: dims (npx+2, npy+2, npz+2), box (34, 10, 1).  Reads past the
// x/y extent of the last tiles are zero-filled by the TMA unit and never used.
CUtensorMap field_map(void* base, int64_t nx, int64_t ny, int64_t nz, int64_t pitch, int64_t plane,
                      cuuint32_t box_x, cuuint32_t box_y, CUtensorMapDataType type, size_t esize) {
    CUtensorMap m;
    const cuuint64_t dims[3] = {(cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nz};
    const cuuint64_t strides[2] = {(cuuint64_t)(pitch * esize), (cuuint64_t)(plane * esize)};
    const cuuint32_t box[3] = {box_x, box_y, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = encode_fn()(&m, type, 3, base, dims, strides, box, estr,
                             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw Error(R3D_ECUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
    return m;
}

}  // namespace r3dg

namespace {

__global__ void totals_kernel(r3dk::Geometry g, r3dk::Physics ph, FieldSet fs, r3dk::Scalars* sc) {
    const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
    double m = 0.0, e = 0.0;
    if (i <= g.npx && j <= g.npy) {
        for (int k = 1 + blockIdx.z; k <= g.npz; k += gridDim.z) {
            const int64_t n = (int64_t)k * g.plane + (int64_t)j * g.pitch + i;
            const double ru = fs.xin[0][n], rv = fs.xin[1][n], rw = fs.xin[2][n];
            const double ro = fs.xin[3][n], tt = fs.xin[4][n];
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

// FP32-bulk state <-> the reference layout in FP64: dev32 (pitched) = (float)(host - bg[k]) on
// upload, host = bg[k] + (double)dev32 on download, for one field of nx*ny*nz cells.  bg is the
// static background column (rho or T), or null for the momenta.
__global__ void to_fp32_kernel(float* out, int64_t pitch, int64_t plane, const double* in, int64_t nx,
                               int64_t ny, int64_t nz, const double* bg) {
    const int64_t n = nx * ny * nz;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = c % nx, j = (c / nx) % ny, k = c / (nx * ny);
        out[k * plane + j * pitch + i] = (float)(in[c] - (bg ? bg[k] : 0.0));
    }
}
__global__ void from_fp32_kernel(double* out, const float* in, int64_t pitch, int64_t plane, int64_t nx,
                                 int64_t ny, int64_t nz, const double* bg) {
    const int64_t n = nx * ny * nz;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = c % nx, j = (c / nx) % ny, k = c / (nx * ny);
        out[c] = (bg ? bg[k] : 0.0) + (double)in[k * plane + j * pitch + i];
    }
}

// Initial condition on the device (src/static_ic.cpp:24-161), one field in the reference layout
// (contiguous nx*ny*nz, local planes): kind 0 zero (momenta, By, Bz), 1 the temperature column,
// 2 the density column (with LMAG less Bx^2/T*obeta, the layer correction, on the domain's
// interior planes: local plane k is global plane z0 + k of nzg), 3 the magnetic layer Bx.  Every
// cell of a plane, x/y ghosts included, takes the plane's value, as the host set-up leaves them
// after its periodic ghost copy.
__global__ void ic_field_kernel(double* out, int64_t nx, int64_t ny, int64_t nz, int kind, const double* col_t,
                                const double* col_r, const double* bfac, double obeta, int lmag, int64_t z0,
                                int64_t nzg) {
    const int64_t n = nx * ny * nz;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = c / (nx * ny);
        double v = 0.0;
        if (kind == 1) {
            v = col_t[k];
        } else if (kind == 2) {
            v = col_r[k];
            if (lmag && z0 + k >= 1 && z0 + k <= nzg - 2)
                v = v - bfac[k] * bfac[k] / col_t[k] * obeta;  // src/static_ic.cpp:104-107
        } else if (kind == 3) {
            v = bfac[k];
        }
        out[c] = v;
    }
}

// Temperature perturbation of one interior plane (src/static_ic.cpp:114-159): T *= 1 + ampt *
// (u - 0.5) with u the plane's RAN2 draws in (j, i) order over the interior cells.
__global__ void ic_perturb_kernel(double* plane, const double* u, int64_t nx, int64_t ny, double ampt) {
    const int64_t npx = nx - 2, n = npx * (ny - 2);
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = 1 + c % npx, j = 1 + c / npx;
        const double w = 1.0 + ampt * (u[c] - 0.5);
        plane[j * nx + i] *= w;
    }
}

// Periodic x/y ghost cells of every plane from the interior (the result of the host's row-then-
// column ghost copy, src/communicate.cpp:70-168 on one domain).
__global__ void ic_ghost_kernel(double* f, int64_t nx, int64_t ny, int64_t nz) {
    const int64_t ring = 2 * nx + 2 * (ny - 2), n = ring * nz;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = c / ring, r = c % ring;
        int64_t i, j;
        if (r < nx) { i = r; j = 0; }
        else if (r < 2 * nx) { i = r - nx; j = ny - 1; }
        else if (r < 2 * nx + (ny - 2)) { i = 0; j = 1 + (r - 2 * nx); }
        else { i = nx - 1; j = 1 + (r - 2 * nx - (ny - 2)); }
        const int64_t si = i == 0 ? nx - 2 : (i == nx - 1 ? 1 : i);
        const int64_t sj = j == 0 ? ny - 2 : (j == ny - 1 ? 1 : j);
        f[(k * ny + j) * nx + i] = f[(k * ny + sj) * nx + si];
    }
}

// RK accumulator of the FP32-bulk form (stored one column left: element (i,j,k) at
// k*plane + j*pitch + i - 1) to the reference layout in FP64, interior columns only (i = 0: 0).
__global__ void z_from_fp32_kernel(double* out, const float* in, int64_t pitch, int64_t plane, int64_t nx,
                                   int64_t ny, int64_t nz, const double* bg) {
    const int64_t n = nx * ny * nz;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n; c += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = c % nx, j = (c / nx) % ny, k = c / (nx * ny);
        out[c] = i == 0 ? 0.0 : (bg ? bg[k] : 0.0) + (double)in[k * plane + j * pitch + i - 1];
    }
}

// Estimated length of one stage launch over `tiles` column tiles x z-chunks of depth k, in
// plane loads: list scheduling of the CTAs in launch order (the chunk is the slowest block
// index, so the last chunk's CTAs run last) onto `slots` resident CTA slots, each CTA costing
// its planes plus the two halo planes.
double launch_estimate(int64_t tiles, int nloc, int k, int64_t slots) {
    std::priority_queue<double, std::vector<double>, std::greater<double>> free_at;
    for (int64_t s = 0; s < slots; ++s) free_at.push(0.0);
    double end = 0.0;
    for (int z0 = 0; z0 < nloc; z0 += k) {
        const double cost = std::min(k, nloc - z0) + 2;
        for (int64_t t = 0; t < tiles; ++t) {
            const double e = free_at.top() + cost;
            free_at.pop();
            free_at.push(e);
            end = std::max(end, e);
        }
    }
    return end;
}

// Chunk depth of a multi-wave launch.  When the depth d divides the planes, the partial last
// wave is full-depth CTAs and leaves most SMs idle for a whole CTA time; a slightly shallower
// depth (at most one chunk more) with a short last chunk fills that tail.  Candidates d down to
// 3d/4; d is kept unless the estimate improves by 0.5%, and the deepest candidate within 0.5%
// of the best is taken (fewer halo planes).  504x504x512 FP64 on B200: 64 -> 62 planes; depths
// 56 and 63 there measured 15.84-15.90 ms per step against 15.98-16.25 ms at 64.
int plan_chunk_depth(int64_t tiles, int nloc, int d, int64_t slots) {
    const int n0 = (nloc + d - 1) / d;
    const double base = launch_estimate(tiles, nloc, d, slots);
    std::vector<std::pair<int, double>> cand;
    for (int k = d; k >= (3 * d + 3) / 4 && k >= 1; --k) {
        if ((nloc + k - 1) / k > n0 + 1) break;
        cand.emplace_back(k, launch_estimate(tiles, nloc, k, slots));
    }
    double best = base;
    for (const auto& c : cand) best = std::min(best, c.second);
    if (best > base * 0.995) return d;
    for (const auto& c : cand)
        if (c.second <= best * 1.005) return c.first;
    return d;
}

// z-chunk depth (planes per CTA) of the stage kernels of a handle over nloc local planes, given
// its precision, FP64 column-tile rows and the device's SM count; R3D_KCHUNK=<planes> in the
// environment overrides it.
int stage_chunk_depth(const r3d_params& p, bool fp32, int tile_rows, int nloc, int num_sms) {
    int depth = nloc >= 512 ? 64 : (nloc >= 256 ? 32 : 16);
    // column tiles of the stage kernel (32 x rows) and its resident CTAs per SM
    unsigned tbx = 0, tby = 0;
    if (fp32) r3dk::stage_fp32_box(&tbx, &tby);
    else r3dk::stage_fp64_box(tile_rows, &tbx, &tby);
    const int64_t tiles = (int64_t)((p.npx + 31) / 32) * ((p.npy + (int)tby - 3) / ((int)tby - 2));
    const int64_t slots = (int64_t)num_sms * (fp32 ? r3dk::stage_fp32_ctas_per_sm()
                                                   : r3dk::stage_fp64_ctas_per_sm(p.lmag, (int)tby - 2));
    if (p.lmag && tby == 8) {
        // 32x6 MHD tiles, two CTAs per SM: 12-plane chunks.  Measured on B200 against the
        // earlier 16/32-plane choice: 126x126x256 0.962 -> 0.922 ms per step, 252x252x256
        // 3.24 -> 3.14-3.17 ms for any depth in 13..24 (10..13 all within 0.6%).
        depth = 12;
    } else if (p.lmag) {
        // few, heavy CTAs: prefer enough z-chunks for >= 4 full waves
        while (depth > 16 && tiles * ((nloc + depth - 1) / depth) < 4 * slots) depth /= 2;
    }
    {
        // small grids, whose launch does not fill the GPU once: the chunk depth (down to 4)
        // that minimises waves x (planes loaded per chunk)
        auto ctas = [&](int k) { return tiles * ((nloc + k - 1) / k); };
        auto cost = [&](int k) { return (ctas(k) + slots - 1) / slots * (k + 2); };
        if (ctas(depth) < slots) {
            int best = depth;
            for (int k = depth / 2; k >= 4; k /= 2)
                if (cost(k) < cost(best)) best = k;
            depth = best;
        } else if (!p.lmag && ctas(depth) <= 64 * slots) {
            depth = plan_chunk_depth(tiles, nloc, depth, slots);
        }
    }
    // R3D_KCHUNK=<planes> overrides the z-chunk depth of the stage kernels (tuning): a whole
    // decimal number, clamped to [1, nloc]; anything else is ignored with a note on stderr
    if (const char* e = getenv("R3D_KCHUNK")) {
        char* end = nullptr;
        errno = 0;
        const long v = strtol(e, &end, 10);
        if (end == e || *end != '\0' || errno == ERANGE || v < 1) {
            fprintf(stderr, "r3d: R3D_KCHUNK='%s' is not a positive whole number; ignored\n", e);
        } else {
            const int k = (int)std::min<long>(v, nloc);
            if (k != depth) fprintf(stderr, "r3d: R3D_KCHUNK overrides the z-chunk depth: %d planes (planned %d)\n", k, depth);
            depth = k;
        }
    }
    return depth;
}

}  // namespace

namespace r3dk {
cudaError_t launch_totals(const Geometry& g, const Physics& ph, const FieldSet& fs, Scalars* sc,
                          cudaStream_t st) {
    dim3 block(32, 8, 1);
    dim3 grid((g.npx + 31) / 32, (g.npy + 7) / 8, (unsigned)std::min(g.npz, 64));
    totals_kernel<<<grid, block, 0, st>>>(g, ph, fs, sc);
    return cudaGetLastError();
}
}  // namespace r3dk

namespace r3dg {

FieldSet fieldset(const r3d_gpu* g) {
    FieldSet fs{};
    for (int q = 0; q < r3dk::kMaxFields; ++q) {
        fs.xin[q] = g->X[g->cur][q];
        fs.xout[q] = g->X[1 - g->cur][q];
        fs.z[q] = g->Z[q];
    }
    return fs;
}

r3dk::FieldSet32 fieldset32(const r3d_gpu* g) {
    r3dk::FieldSet32 fs{};
    for (int q = 0; q < 5; ++q) {
        fs.xin[q] = g->X32[g->cur][q];
        fs.xout[q] = g->X32[1 - g->cur][q];
        fs.z[q] = g->Z32[q];
    }
    return fs;
}

// R(k), T0(k) over the global z index: ghost 0 -> T(0), interior k -> T(k-1), ghost npz+1 -> the
// bottom value (src/static_ic.cpp:53-89 stitched over ranks); for a z slab, the nloc+2 planes
// from global plane z0 on.
void background_columns(const r3d_gpu* g, std::vector<double>& R, std::vector<double>& T) {
    const r3d_params& p = g->p;
    std::vector<double> t, r;
    static_profile(p, t, r);
    const int nz = p.npz + 2, nl = g->nloc + 2;
    R.assign(nl, 0.0);
    T.assign(nl, 0.0);
    for (int k = 0; k < nl; ++k) {
        const int kg = g->z0 + k;
        const int src = kg == 0 ? 0 : (kg == nz - 1 ? p.npz - 1 : kg - 1);
        R[k] = r[src];
        T[k] = t[src];
    }
}

// A temporary FP64 field in the reference layout plus the rho / T background columns on the
// device, for the FP32-bulk upload and download (freed when it goes out of scope, after the
// stream has drained).
struct Fp64Staging {
    r3d_gpu* g;
    size_t n = 0;
    double* buf = nullptr;
    double* cols = nullptr;  // R[nz], T[nz]
    explicit Fp64Staging(r3d_gpu* gg) : g(gg) {
        const Derived& d = g->d;
        n = (size_t)d.nx * d.ny * d.nz;
        std::vector<double> R, T;
        background_columns(g, R, T);
        cuda_ok(cudaMalloc(&buf, n * sizeof(double)), "cudaMalloc(staging)");
        cuda_ok(cudaMalloc(&cols, 2 * R.size() * sizeof(double)), "cudaMalloc(staging)");
        R.insert(R.end(), T.begin(), T.end());
        cuda_ok(cudaMemcpyAsync(cols, R.data(), R.size() * sizeof(double), cudaMemcpyHostToDevice, g->stream),
                "staging columns");
        cuda_ok(cudaStreamSynchronize(g->stream), "staging columns");  // R is a host temporary
    }
    ~Fp64Staging() {
        cudaStreamSynchronize(g->stream);
        cudaFree(buf);
        cudaFree(cols);
    }
    Fp64Staging(const Fp64Staging&) = delete;
    Fp64Staging& operator=(const Fp64Staging&) = delete;
    const double* bg(int q) const { return q == 3 ? cols : (q == 4 ? cols + g->d.nz : nullptr); }
    unsigned blocks() const { return (unsigned)std::min<size_t>((n + 255) / 256, 148 * 16); }
};

double plume_tpr(const r3d_gpu* g) {
    const double timt = g->host_timc + g->host_timi;  // src/bcon.cpp:22
    return (g->p.tc != 0.0) ? g->p.tp + (1.0 - g->p.tp) * std::exp(-timt / g->p.tc) : g->p.tp;
}

// The time factor of the embedded heat loss (itcon 2), 3dmhdsub.f:1801-1818: TP*OCV, ramped by
// 0.5*(1 + tanh(log(3)/QFH*(TIMT - TC))) when TC != 0; LOG(3.0E00) is a single-precision literal.
double heat_prefix(const r3d_gpu* g) {
    const r3d_params& p = g->p;
    const double tpocv = p.tp * g->ph.ocv;
    if (p.tc == 0.0) return tpocv;
    const double timt = g->host_timc + g->host_timi;
    return tpocv * 0.5 * (1.0 + std::tanh((double)logf(3.0f) / p.qfh * (timt - p.tc)));
}

void launch_dt_full_any(r3d_gpu* g, int only_refold) {
    if (g->fp32)
        cuda_ok(r3dk::launch_dt_full_fp32(g->geo, g->ph, g->lines, g->bg, fieldset32(g), g->dsc, g->stream,
                                          only_refold),
                "dt_full32");
    else
        cuda_ok(r3dk::launch_dt_full(g->geo, g->ph, g->lines, fieldset(g), g->dsc, g->stream, only_refold),
                "dt_full");
}

// Density diffusion: the horizontal means of rho (and WWZ for ID 1) of the stage's input state,
// into the line buffer the stage kernel reads them from.
void launch_plane_mean(r3d_gpu* g, const FieldSet& fs) {
    cuda_ok(r3dk::launch_plane_mean(g->geo, fs.xin[3], const_cast<double*>(g->lines.rom),
                                    const_cast<double*>(g->lines.wwz), g->ph.id_mode, g->stream),
            "plane_mean");
}

// Queue one step (nstages substages) on the device.
void enqueue_step_begin(r3d_gpu* g) {
    Range r("r3d.step_begin");
    g->bnd.tpr = plume_tpr(g);
    if (g->ph.heat_on) g->ph.heat_pre = heat_prefix(g);
    if (g->halo) halo_reduce_limits(g);
    cuda_ok(r3dk::launch_step_begin(g->ph, g->dsc, g->stream), "step_begin");
}

void enqueue_stage(r3d_gpu* g, int s) {
    Range r("r3d.stage");
    if (g->fp32) {
        r3dk::FieldSet32 fs = fieldset32(g);
        cuda_ok(r3dk::launch_stage_fp32(s, g->maps[g->cur], g->geo, g->ph, g->lines, g->bg, fs, g->dsc,
                                        g->kchunk, g->stream),
                "stage32");
        cuda_ok(r3dk::launch_bcon_fp32(g->geo, g->ph, g->lines, g->bnd, g->bg, fs, g->dsc, s == 2 ? 1 : 0, g->stream),
                "bcon32");
    } else {
        FieldSet fs = fieldset(g);
        if (g->ph.id_mode) launch_plane_mean(g, fs);
        cuda_ok(r3dk::launch_stage_fp64(s, g->maps[g->cur], g->geo, g->ph, g->lines, fs, g->dsc, g->kchunk, g->stream),
                "stage");
        cuda_ok(r3dk::launch_bcon(g->geo, g->ph, g->lines, g->bnd, fs, g->dsc, s == 2 ? 1 : 0, g->stream), "bcon");
    }
    g->cur = 1 - g->cur;
}

void enqueue_step_end(r3d_gpu* g, int nstages) {
    Range r("r3d.step_end");
    cuda_ok(r3dk::launch_step_end(g->dsc, g->stream, nstages == 3 ? 1 : 0), "step_end");
    if (nstages < 3) launch_dt_full_any(g);  // the next dt needs the limits of this partial-step state
    else if (g->dt_filter) launch_dt_full_any(g, 1);  // only if the filtered limits failed the check
}

// Queue one step (nstages substages) on the device; with a Halo, the dt keys are reduced over
// the slabs before the step and the ghost planes exchanged after every stage.
void enqueue_step(r3d_gpu* g, int nstages, Timer& tm, int& launches, int& stage_launches) {
    Range step_range("r3d.step");
    g->bnd.tpr = plume_tpr(g);
    if (g->ph.heat_on) g->ph.heat_pre = heat_prefix(g);
    tm.begin();
    if (g->halo) halo_reduce_limits(g);
    cuda_ok(r3dk::launch_step_begin(g->ph, g->dsc, g->stream), "step_begin");
    tm.end(2);
    ++launches;
    for (int s = 0; s < nstages; ++s) {
        Range stage_range("r3d.stage");
        tm.begin();
        if (g->fp32) {
            r3dk::FieldSet32 fs = fieldset32(g);
            cuda_ok(r3dk::launch_stage_fp32(s, g->maps[g->cur], g->geo, g->ph, g->lines, g->bg, fs, g->dsc, g->kchunk, g->stream), "stage32");
            tm.end(0);
            tm.begin();
            cuda_ok(r3dk::launch_bcon_fp32(g->geo, g->ph, g->lines, g->bnd, g->bg, fs, g->dsc, s == 2 ? 1 : 0, g->stream), "bcon32");
        } else {
            FieldSet fs = fieldset(g);
            if (g->ph.id_mode) {
                launch_plane_mean(g, fs);
                tm.end(2);
                ++launches;
                tm.begin();
            }
            cuda_ok(r3dk::launch_stage_fp64(s, g->maps[g->cur], g->geo, g->ph, g->lines, fs, g->dsc, g->kchunk, g->stream), "stage");
            tm.end(0);
            tm.begin();
            cuda_ok(r3dk::launch_bcon(g->geo, g->ph, g->lines, g->bnd, fs, g->dsc, s == 2 ? 1 : 0, g->stream), "bcon");
        }
        tm.end(1);
        launches += 2;
        ++stage_launches;
        g->cur = 1 - g->cur;
        if (g->halo) {
            tm.begin();
            halo_exchange(g);
            tm.end(2);
        }
    }
    tm.begin();
    cuda_ok(r3dk::launch_step_end(g->dsc, g->stream, nstages == 3 ? 1 : 0), "step_end");
    ++launches;
    if (nstages < 3) {  // the next dt needs the limits of this (partial-step) state
        launch_dt_full_any(g);
        ++launches;
    } else if (g->dt_filter) {  // re-evaluation, only if the filtered limits failed the check
        launch_dt_full_any(g, 1);
        ++launches;
    }
    tm.end(2);
    g->work_ok = nstages == 3;
}

void* state_field(r3d_gpu* g, int q, size_t* esize) {
    if (g->fp32) {
        *esize = sizeof(float);
        return g->X32[g->cur][q];
    }
    *esize = sizeof(double);
    return g->X[g->cur][q];
}

int state_fields(const r3d_gpu* g) { return g->fp32 ? 5 : g->nfields; }

void pull_scalars(r3d_gpu* g, r3d_scalars* sc) {
    cuda_ok(cudaMemcpyAsync(g->hsc, g->dsc, sizeof(r3dk::Scalars), cudaMemcpyDeviceToHost, g->stream),
            "scalar read-back");
    cuda_ok(cudaStreamSynchronize(g->stream), "step");
    if (g->hsc->err != r3dk::kErrNone)
        throw Error(R3D_ECUDA, "a stage kernel abandoned a bounded TMA wait (error " +
                                   std::to_string(g->hsc->err) + "); the state is invalid");
    g->host_timc = g->hsc->timc;
    g->host_timi = g->hsc->timi;
    if (sc) {
        sc->dt = g->hsc->dt;
        sc->timc = g->hsc->timc;
        sc->timt = g->hsc->timt;
        sc->timi = g->hsc->timi;
        sc->umach = g->hsc->umach;
        sc->tb = g->hsc->tb;
        sc->nit = g->hsc->nit;
    }
}

// The graph of two whole steps for the current buffer parity, captured on first use.  Every
// launch argument of a step is fixed for the handle's lifetime (buffers, TMA maps, physics, the
// boundary set-up when tc == 0); the step-to-step state lives in device memory.
cudaGraphExec_t two_step_graph(r3d_gpu* g) {
    cudaGraphExec_t& ex = g->step_graph[g->cur];
    if (ex) return ex;
    Range r("r3d.capture");
    const int cur0 = g->cur;
    Timer off{g, false, nullptr};
    int l = 0, s = 0;
    cuda_ok(cudaStreamBeginCapture(g->stream, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
    cudaGraph_t graph = nullptr;
    try {
        enqueue_step(g, 3, off, l, s);
        enqueue_step(g, 3, off, l, s);
    } catch (...) {
        cudaStreamEndCapture(g->stream, &graph);
        if (graph) cudaGraphDestroy(graph);
        g->cur = cur0;
        throw;
    }
    cuda_ok(cudaStreamEndCapture(g->stream, &graph), "cudaStreamEndCapture");
    g->cur = cur0;
    const cudaError_t e = cudaGraphInstantiate(&ex, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
        ex = nullptr;
        cuda_ok(e, "cudaGraphInstantiate");
    }
    return ex;
}

void run_steps(r3d_gpu* g, int nsteps, r3d_scalars* sc, r3d_timing* tmout, bool sync) {
    if (!g) throw std::invalid_argument("null handle");
    if (!g->uploaded) throw Error(R3D_ESTATE, "step before upload");
    if (nsteps < 0) throw std::invalid_argument("nsteps < 0");
    DeviceGuard dg(g->device);
    Timer tm{g, tmout != nullptr, tmout};
    int launches = 0, stage_launches = 0;
    int n = 0;
    // Untimed runs without a host dependency replay a two-step CUDA graph (after one step has
    // gone through the eager path, which configures the kernels): on small grids the nine
    // launches per step would otherwise set the pace.
    const bool graphs = !tmout && g->p.tc == 0.0 && !g->halo;
    if (graphs && g->steps_enqueued == 0 && nsteps > 0) {
        enqueue_step(g, 3, tm, launches, stage_launches);
        ++g->steps_enqueued;
        ++n;
    }
    if (graphs && nsteps - n >= 2) {
        cudaGraphExec_t ex = two_step_graph(g);
        for (; n + 2 <= nsteps; n += 2) {
            cuda_ok(cudaGraphLaunch(ex, g->stream), "cudaGraphLaunch");
            g->steps_enqueued += 2;
        }
    }
    for (; n < nsteps; ++n) {
        enqueue_step(g, 3, tm, launches, stage_launches);
        ++g->steps_enqueued;
        if (g->p.tc != 0.0 && n + 1 < nsteps) pull_scalars(g, nullptr);  // host clock for BCON
    }
    if (nsteps > 0) g->work_ok = true;
    if (sync || tmout) pull_scalars(g, sc);
    if (tmout) {
        std::memset(tmout, 0, sizeof(*tmout));
        for (auto& sp : tm.spans) {
            float ms = 0.f;
            cuda_ok(cudaEventElapsedTime(&ms, g->ev[sp.first], g->ev[sp.first + 1]), "event time");
            if (sp.second == 0) tmout->stage_ms += ms;
            else if (sp.second == 1) tmout->bcon_ms += ms;
            else tmout->other_ms += ms;
        }
        if (!tm.spans.empty()) {
            float ms = 0.f;
            cuda_ok(cudaEventElapsedTime(&ms, g->ev[tm.spans.front().first], g->ev[tm.spans.back().first + 1]),
                    "event time");
            tmout->total_ms = ms;
        }
        tmout->stage_launches = stage_launches;
        tmout->total_launches = launches;
    }
}

void upload_lines(r3d_gpu* g, const r3d_host_state* st) {
    const r3d_params& p = g->p;
    const Derived& d = g->d;
    const int64_t NX = d.nx, NY = d.ny, NZ = d.nz;
    // host tables (products keep the reference association)
    std::vector<double> dxxdx(st->dxxdx, st->dxxdx + NX), d2xxdx2(st->d2xxdx2, st->d2xxdx2 + NX),
        ddx(st->ddx, st->ddx + NX);
    std::vector<double> dyydy(st->dyydy, st->dyydy + NY), ddy(st->ddy, st->ddy + NY),
        d2yydy2(st->d2yydy2, st->d2yydy2 + NY);
    std::vector<double> tmpy(NY), tmpy1(NY), tmpy2(NY);
    for (int64_t j = 0; j < NY; ++j) {
        tmpy[j] = d.hy * st->dyydy[j];                       // src/fluxes.cpp:90
        tmpy1[j] = d.hy * st->d2yydy2[j];                    // src/fluxes.cpp:253
        tmpy2[j] = d.h2y * st->dyydy[j] * st->dyydy[j];      // src/fluxes.cpp:254
    }
    std::vector<double> dzzdz(st->dzzdz, st->dzzdz + NZ), d2zzdz2(st->d2zzdz2, st->d2zzdz2 + NZ),
        ddz(st->ddz, st->ddz + NZ), rkapa(st->rkapa, st->rkapa + NZ), dkapa(st->dkapa, st->dkapa + NZ);
    std::vector<double> tmpz(NZ), tmpz1(NZ), tmpz2(NZ);
    for (int64_t k = 0; k < NZ; ++k) {
        tmpz[k] = d.hz * st->dzzdz[k];                       // src/fluxes.cpp:101
        tmpz1[k] = d.hz * st->d2zzdz2[k];                    // src/fluxes.cpp:250
        tmpz2[k] = d.h2z * st->dzzdz[k] * st->dzzdz[k];      // src/fluxes.cpp:251
    }
    // plume profile factors (src/bcon.cpp:47-68); host libm, as the reference
    std::vector<double> px(NX, 0.0), py(NY, 0.0);
    const double cln = (double)(-4.0f * logf(2.0f)) / (p.hh * p.hh);
    for (int64_t i = 0; i < NX; ++i) {
        const double a = st->exx[i] - p.xp;
        px[i] = (p.itcon == 0) ? std::exp(cln * a * a) : std::exp(cln * (a * a));
    }
    for (int64_t j = 0; j < NY; ++j) {
        const double a = st->wyy[j] - p.yp;
        py[j] = (p.itcon == 0) ? std::exp(cln * a * a) : std::exp(cln * (a * a));
    }
    // embedded heat loss profiles (itcon 2, 3dmhdsub.f:1800,1806-1809): the Fortran's
    // CLN=-4.0E00*LOG(2.0E00)/HH/HH (single-precision literal, then two divisions) and
    // EXP(CLN*(EXX(I)-XP)**2) with x**2 = x*x; host libm
    std::vector<double> hx_(NX, 0.0), hy_(NY, 0.0), hz_(NZ, 0.0);
    if (p.itcon == 2) {
        const double clh = (double)(-4.0f * logf(2.0f)) / p.hh / p.hh;
        for (int64_t i = 0; i < NX; ++i) {
            const double a = st->exx[i] - p.xp;
            hx_[i] = std::exp(clh * (a * a));
        }
        for (int64_t j = 0; j < NY; ++j) {
            const double a = st->wyy[j] - p.yp;
            hy_[j] = std::exp(clh * (a * a));
        }
        for (int64_t k = 0; k < NZ; ++k) {
            const double a = st->zee[k] - p.zp;
            hz_[k] = std::exp(clh * (a * a));
        }
    }
    // density diffusion (ID 1, 2; 3dmhdsub.f:1337-1344): the per-plane horizontal means of rho
    // (written on the device before each stage) and WWZ, for ID 2 the Fortran's
    // EXP(CLN*ZEE**2)+EXP(CLN*(ZEE-ZMAX)**2) with SGM=0.1E00, CLN=-4.0E00*LOG(2.0E00)/SGM/SGM
    // (single-precision literals); host libm.  ID 1: WWZ = 1/ROM, written with the means.
    std::vector<double> rom_(NZ, 0.0), wwz_(NZ, 0.0);
    if (p.id == 2) {
        const double sgm = (double)0.1f;
        const double cln = (double)(-4.0f * logf(2.0f)) / sgm / sgm;
        for (int64_t k = 0; k < NZ; ++k) {
            const double z = st->zee[k], zm = st->zee[k] - p.zmax;
            wwz_[k] = std::exp(cln * (z * z)) + std::exp(cln * (zm * zm));
        }
    }
    std::vector<const std::vector<double>*> tabs = {&dxxdx, &d2xxdx2, &ddx,  &dyydy, &tmpy,
                                                    &tmpy1, &tmpy2,   &ddy,  &dzzdz, &d2zzdz2,
                                                    &tmpz,  &tmpz1,   &tmpz2, &ddz,  &rkapa,
                                                    &dkapa, &px,      &py,   &d2yydy2, &hx_,
                                                    &hy_,   &hz_,     &rom_, &wwz_};
    size_t total = 0;
    for (auto* t : tabs) total += (t->size() + 15) / 16 * 16;
    if (!g->line_buf) {
        cuda_ok(cudaMalloc(&g->line_buf, total * sizeof(double)), "cudaMalloc(lines)");
        g->bytes += total * sizeof(double);
    }
    std::vector<double> packed(total, 0.0);
    std::vector<const double*> dev;
    size_t off = 0;
    for (auto* t : tabs) {
        std::memcpy(packed.data() + off, t->data(), t->size() * sizeof(double));
        dev.push_back(g->line_buf + off);
        off += (t->size() + 15) / 16 * 16;
    }
    cuda_ok(cudaMemcpy(g->line_buf, packed.data(), total * sizeof(double), cudaMemcpyHostToDevice),
            "upload lines");
    r3dk::Lines& L = g->lines;
    L.dxxdx = dev[0]; L.d2xxdx2 = dev[1]; L.ddx = dev[2];
    L.dyydy = dev[3]; L.tmpy = dev[4]; L.tmpy1 = dev[5]; L.tmpy2 = dev[6]; L.ddy = dev[7];
    L.dzzdz = dev[8]; L.d2zzdz2 = dev[9]; L.tmpz = dev[10]; L.tmpz1 = dev[11]; L.tmpz2 = dev[12];
    L.ddz = dev[13]; L.rkapa = dev[14]; L.dkapa = dev[15]; L.plume_x = dev[16]; L.plume_y = dev[17];
    L.d2yydy2 = dev[18];
    L.heat_x = dev[19]; L.heat_y = dev[20]; L.heat_z = dev[21];
    L.rom = dev[22]; L.wwz = dev[23];
    g->ph.id_mode = p.id;
    g->ph.id_dh = p.dh;
    g->ph.id_dv = p.dv;
    g->ph.id_dh_ore = p.dh * d.ore;  // TMP = DH*ORE*WWZ(K) (3dmhdsub.f:1363, 1380)
    g->ph.id_dv_ore = p.dv * d.ore;
    g->ph.heat_on = p.itcon == 2 ? 1 : 0;
    g->ph.hh = p.hh;
    g->ph.hh_one = p.hh == 1.0 ? 1 : 0;
    g->ph.heat_pre = heat_prefix(g);
    bool kc = true;
    for (int64_t k = 1; k <= NZ - 2; ++k) kc = kc && rkapa[k] == 1.0 && dkapa[k] == 0.0;
    g->ph.kappa_const = kc ? 1 : 0;
    const double dzs = (double)(1.0f / (float)(p.npz - 1));
    g->bnd.dz_top = dzs / st->dzzdz[1];            // src/bcon.cpp:59
    g->bnd.dz_bot = dzs / st->dzzdz[NZ - 2];       // src/bcon.cpp:124 (plane npz of the domain)
}

// FP32-bulk background tables (see r3dk::Background).
void upload_background(r3d_gpu* g, const r3d_host_state* st) {
    const r3d_params& p = g->p;
    const Derived& d = g->d;
    const int64_t NZ = d.nz;
    std::vector<double> R, T;
    background_columns(g, R, T);
    std::vector<double> hres(NZ, 0.0), dt0(NZ, 0.0), lt0(NZ, 0.0);
    for (int64_t k = 1; k < NZ - 1; ++k) {
        const double tz = d.hz * st->dzzdz[k];
        const double tz1 = d.hz * st->d2zzdz2[k];
        const double tz2 = d.h2z * st->dzzdz[k] * st->dzzdz[k];
        hres[k] = p.grav * R[k] - (R[k + 1] * T[k + 1] - R[k - 1] * T[k - 1]) * tz;
        dt0[k] = T[k + 1] - T[k - 1];
        lt0[k] = dt0[k] * tz1 + (T[k + 1] - 2.0 * T[k] + T[k - 1]) * tz2;
    }
    const size_t nd = (size_t)NZ, pad = (nd + 15) / 16 * 16;
    const size_t bytes = pad * (5 * sizeof(double) + 2 * sizeof(float)) + nd * 12 * sizeof(float);
    if (!g->bg_buf) {
        cuda_ok(cudaMalloc(&g->bg_buf, bytes), "cudaMalloc(background)");
        g->bytes += bytes;
    }
    std::vector<unsigned char> host(bytes, 0);
    double* hd = reinterpret_cast<double*>(host.data());
    const std::vector<double>* cols[5] = {&R, &T, &hres, &dt0, &lt0};
    for (int c = 0; c < 5; ++c) std::memcpy(hd + c * pad, cols[c]->data(), nd * sizeof(double));
    float* hf = reinterpret_cast<float*>(hd + 5 * pad);
    for (size_t k = 0; k < nd; ++k) {
        hf[k] = (float)R[k];
        hf[pad + k] = (float)T[k];
    }
    float* kf = hf + 2 * pad;  // 12 floats per plane (3 x float4), 16-byte aligned
    for (size_t k = 0; k < nd; ++k) {
        float* e = kf + 12 * k;
        e[0] = (float)(d.hz * st->dzzdz[k]);
        e[1] = (float)(d.hz * st->d2zzdz2[k]);
        e[2] = (float)(d.h2z * st->dzzdz[k] * st->dzzdz[k]);
        e[3] = (float)(d.hz * st->dzzdz[k]);
        e[4] = (float)hres[k];
        e[5] = (float)dt0[k];
        e[6] = (float)lt0[k];
        e[7] = (float)st->rkapa[k];
        e[8] = (float)st->dkapa[k];
        e[9] = (float)R[k];
        e[10] = (float)T[k];
        e[11] = 0.0f;
    }
    cuda_ok(cudaMemcpy(g->bg_buf, host.data(), host.size(), cudaMemcpyHostToDevice), "upload background");
    const double* dd = static_cast<const double*>(g->bg_buf);
    const float* df = reinterpret_cast<const float*>(dd + 5 * pad);
    g->bg.r = dd;
    g->bg.t = dd + pad;
    g->bg.hres = dd + 2 * pad;
    g->bg.dt0 = dd + 3 * pad;
    g->bg.lt0 = dd + 4 * pad;
    g->bg.rf = df;
    g->bg.tf = df + pad;
    g->bg.kf = reinterpret_cast<const float4*>(df + 2 * pad);
}

}  // namespace r3dg

namespace r3dg {

// A handle over global planes z0+1 .. z0+nloc (the whole domain: z0 = 0, nloc = npz); its host
// and device arrays hold nloc+2 planes, the outer two being the z neighbours' planes (or the
// domain's constant ghost planes).  With shared_stream the handle launches on that stream and
// does not own it.
r3d_gpu* create_handle(const r3d_params& pin, int z0, int nloc, cudaStream_t shared_stream) {
    const r3d_params* p = &pin;
    check_params(*p);
    if (z0 < 0 || nloc < 4 || z0 + nloc > p->npz)
        throw std::invalid_argument("a z slab needs 4 <= nloc and z0 + nloc <= npz");
    auto g = new r3d_gpu();
    try {
            g->p = *p;
            g->d = derive(*p);
            g->z0 = z0;
            g->nloc = nloc;
            g->d.nz = nloc + 2;  // planes held here (global extents stay in p)
            g->device = p->gpu_id;
            int ndev = 0;
            cuda_ok(cudaGetDeviceCount(&ndev), "cudaGetDeviceCount");
            if (g->device < 0 || g->device >= ndev) throw std::invalid_argument("--gpu id out of range");
            DeviceGuard dg(g->device);
            if (shared_stream) {
                g->stream = shared_stream;
                g->own_stream = false;
            } else {
                cuda_ok(cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking), "cudaStreamCreate");
            }
            const Derived& d = g->d;
            g->nfields = p->lmag ? 8 : 5;
            g->geo.npx = p->npx;
            g->geo.npy = p->npy;
            g->geo.npz = nloc;
            g->geo.top_edge = z0 == 0 ? 1 : 0;
            g->geo.bot_edge = z0 + nloc == p->npz ? 1 : 0;
            cuda_ok(cudaDeviceGetAttribute(&g->num_sms, cudaDevAttrMultiProcessorCount, g->device),
                    "cudaDeviceGetAttribute(multiprocessors)");
            g->geo.tile_rows = r3dk::stage_fp64_rows(p->lmag, p->npx, p->npy, nloc, g->num_sms);
            g->geo.pitch = (d.nx + 15) / 16 * 16;
            g->geo.plane = g->geo.pitch * d.ny;
            if (g->geo.plane * d.nz >= (int64_t(1) << 31))
                throw std::invalid_argument("grid too large: a field must hold fewer than 2^31 elements");
            g->fp32 = p->precision == R3D_PREC_FP32BULK;
            if (g->fp32) {
                g->geo.pitch = (d.nx + 31) / 32 * 32;  // 128-byte rows of floats
                g->geo.plane = g->geo.pitch * d.ny;
                const size_t nb = (size_t)g->geo.plane * d.nz * sizeof(float);
                for (int b = 0; b < 2; ++b)
                    for (int q = 0; q < 5; ++q) {
                        cuda_ok(cudaMalloc(&g->X32[b][q], nb), "cudaMalloc(state32)");
                        g->bytes += nb;
                    }
                for (int q = 0; q < 5; ++q) {
                    cuda_ok(cudaMalloc(&g->Z32[q], nb), "cudaMalloc(accumulator32)");
                    cuda_ok(cudaMemsetAsync(g->Z32[q], 0, nb, g->stream), "cudaMemset");
                    g->bytes += nb;
                }
                unsigned bx = 0, by = 0;
                r3dk::stage_fp32_box(&bx, &by);
                for (int b = 0; b < 2; ++b)
                    for (int q = 0; q < 5; ++q)
                        g->maps[b].m[q] = field_map(g->X32[b][q], d.nx, d.ny, d.nz, g->geo.pitch, g->geo.plane,
                                                    bx, by, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, sizeof(float));
            } else {
                const size_t nbytes = (size_t)g->geo.plane * d.nz * sizeof(double);
                for (int b = 0; b < 2; ++b)
                    for (int q = 0; q < g->nfields; ++q) {
                        cuda_ok(cudaMalloc(&g->X[b][q], nbytes), "cudaMalloc(state)");
                        g->bytes += nbytes;
                    }
                unsigned bx = 0, by = 0;
                r3dk::stage_fp64_box(g->geo.tile_rows, &bx, &by);  // the box the stage kernel expects per plane
                for (int b = 0; b < 2; ++b)
                    for (int q = 0; q < g->nfields; ++q)
                        g->maps[b].m[q] = field_map(g->X[b][q], d.nx, d.ny, d.nz, g->geo.pitch, g->geo.plane,
                                                    bx, by, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, sizeof(double));
                for (int q = 0; q < g->nfields; ++q) {
                    cuda_ok(cudaMalloc(&g->Z[q], nbytes), "cudaMalloc(accumulator)");
                    cuda_ok(cudaMemsetAsync(g->Z[q], 0, nbytes, g->stream), "cudaMemset");
                    g->bytes += nbytes;
                }
            }
            cuda_ok(cudaMalloc(&g->dsc, sizeof(r3dk::Scalars)), "cudaMalloc(scalars)");
            cuda_ok(cudaMallocHost(&g->hsc, sizeof(r3dk::Scalars)), "cudaMallocHost");
            r3dk::Physics& ph = g->ph;
            ph.hx = d.hx; ph.h2x = d.h2x; ph.hy = d.hy; ph.hz = d.hz; ph.h2y = d.h2y; ph.h2z = d.h2z;
            ph.tmag = d.obeta * d.orm * d.ocv;  // 3dmhdsub.f:2308
            ph.c13 = d.c13; ph.c23 = d.c23; ph.c43 = d.c43; ph.ore = d.ore; ph.ocv = d.ocv;
            ph.grav = p->grav;
            ph.tdiff = d.ocv / d.repr;
            ph.theat = d.ocv * d.ore;
            ph.theat43 = d.c43 * d.ocv * d.ore;
            ph.t13 = d.c13 * d.ore;
            ph.omx = d.omx; ph.omz = d.omz;
            ph.gamma = p->gamma; ph.ogamma = 1.0 / p->gamma; ph.re = p->re; ph.repr = d.repr;
            ph.cv = d.cv; ph.rm = p->rm; ph.obeta = d.obeta; ph.orm = d.orm; ph.sff = p->sf;
            for (int s = 0; s < 3; ++s) { ph.gam[s] = d.gam[s]; ph.zeta[s] = d.zeta[s]; }
            ph.lrot = p->lrot; ph.lmag = p->lmag;
            ph.kappa_const = 1;
            ph.gamma_f = (float)ph.gamma; ph.ogamma_f = (float)ph.ogamma; ph.obeta_f = (float)ph.obeta;
            r3dk::Boundary& b = g->bnd;
            // 3dmhdsub.f:2807-2887: a plume for itcon 0/1 with tp != 0, else constant T for itcon
            // 0 and 2 (the latter with the embedded heat loss in FLUXES), half-domain T for 4,
            // constant flux for 1
            if (p->tp != 0.0 && (p->itcon == 0 || p->itcon == 1)) b.top_mode = p->itcon == 0 ? 2 : 3;
            else if (p->itcon == 4) b.top_mode = 4;
            else if (p->itcon == 3) b.top_mode = 5;
            else b.top_mode = (p->itcon == 0 || p->itcon == 2) ? 0 : 1;
            g->ph.top_free = p->itcon == 3 ? 1 : 0;
            b.bottom_mode = p->izcon;
            b.hh = p->hh; b.theta = p->theta; b.tp = p->tp; b.tpr = p->tp;
            b.half_nx = (int)(d.nx / 2);
            g->kchunk = stage_chunk_depth(*p, g->fp32, g->geo.tile_rows, nloc, g->num_sms);
            cuda_ok(cudaStreamSynchronize(g->stream), "create");
    } catch (...) {
        destroy_handle(g);
        throw;
    }
    return g;
}

void destroy_handle(r3d_gpu* g) {
    if (!g) return;
    DeviceGuard dg(g->device);
    if (g->stream) cudaStreamSynchronize(g->stream);
    for (auto& ex : g->step_graph)
        if (ex) cudaGraphExecDestroy(ex);
    halo_free(g);
    adjoint_free(g);
    cudaFree(g->fscr);
    for (int b = 0; b < 2; ++b)
        for (int q = 0; q < r3dk::kMaxFields; ++q) cudaFree(g->X[b][q]);
    for (int q = 0; q < r3dk::kMaxFields; ++q) cudaFree(g->Z[q]);
    for (int b = 0; b < 2; ++b)
        for (int q = 0; q < 5; ++q) cudaFree(g->X32[b][q]);
    for (int q = 0; q < 5; ++q) cudaFree(g->Z32[q]);
    cudaFree(g->bg_buf);
    cudaFree(g->line_buf);
    cudaFree(g->dsc);
    if (g->hsc) cudaFreeHost(g->hsc);
    for (auto e : g->ev) cudaEventDestroy(e);
    if (g->stream && g->own_stream) cudaStreamDestroy(g->stream);
    delete g;
}

}  // namespace r3dg

extern "C" {

int r3d_gpu_create(const r3d_params* p, r3d_gpu** out) {
    return guarded([&] {
        if (!p || !out) throw std::invalid_argument("null argument");
        *out = nullptr;
        *out = create_handle(*p, 0, p->npz, nullptr);
    });
}

int r3d_gpu_create_slab(const r3d_params* p, int z0, int nz, r3d_gpu** out) {
    return guarded([&] {
        if (!p || !out) throw std::invalid_argument("null argument");
        *out = nullptr;
        *out = create_handle(*p, z0, nz, nullptr);
    });
}

int r3d_gpu_destroy(r3d_gpu* g) {
    destroy_handle(g);
    return R3D_OK;
}

namespace r3dg {

// Device memory freed when it goes out of scope (after the handle's stream has drained).
struct DeviceBuffer {
    void* p = nullptr;
    cudaStream_t st = nullptr;
    explicit DeviceBuffer(size_t bytes, cudaStream_t s = nullptr) : st(s) { cuda_ok(cudaMalloc(&p, bytes), "cudaMalloc"); }
    ~DeviceBuffer() {
        if (st) cudaStreamSynchronize(st);
        cudaFree(p);
    }
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
};

// The seeded temperature perturbation of the initial condition into t (the handle's planes in
// the reference layout, on the device), then its periodic x/y ghosts.  The RAN2 stream is one
// sequential chain (a shuffle table indexed by the previous draw), so the host draws it plane by
// plane into a ring of pinned buffers while the device copies and applies the planes before.
void perturb_temperature(r3d_gpu* g, double* t) {
    const r3d_params& p = g->p;
    const Derived& d = g->d;
    const int64_t NX = d.nx, NY = d.ny, NZ = d.nz, per = (int64_t)p.npx * p.npy;
    PerturbationDraws draws(p, g->z0, g->nloc);
    constexpr int kRing = 4;
    if (draws.last() >= draws.first()) {
        double* host = nullptr;
        cuda_ok(cudaMallocHost(&host, kRing * per * sizeof(double)), "cudaMallocHost(draws)");
        struct FreeHost {
            double* p;
            ~FreeHost() { cudaFreeHost(p); }
        } free_host{host};
        DeviceBuffer dev(kRing * per * sizeof(double), g->stream);
        cudaEvent_t ev[kRing] = {};
        struct Events {
            cudaEvent_t* e;
            ~Events() {
                for (int s = 0; s < kRing; ++s)
                    if (e[s]) cudaEventDestroy(e[s]);
            }
        } events{ev};
        for (int s = 0; s < kRing; ++s) cuda_ok(cudaEventCreateWithFlags(&ev[s], cudaEventDisableTiming), "event");
        const unsigned blocks = (unsigned)std::min<int64_t>((per + 255) / 256, (int64_t)g->num_sms * 8);
        for (int64_t k = draws.first(), n = 0; k <= draws.last(); ++k, ++n) {
            const int s = (int)(n % kRing);
            double* h = host + s * per;
            double* u = static_cast<double*>(dev.p) + s * per;
            if (n >= kRing) cuda_ok(cudaEventSynchronize(ev[s]), "draw ring");  // plane n - kRing is done
            draws.next_plane(h);
            cuda_ok(cudaMemcpyAsync(u, h, per * sizeof(double), cudaMemcpyHostToDevice, g->stream), "draws");
            ic_perturb_kernel<<<blocks, 256, 0, g->stream>>>(t + k * NX * NY, u, NX, NY, p.ampt);
            cuda_ok(cudaGetLastError(), "ic_perturb_kernel");
            cuda_ok(cudaEventRecord(ev[s], g->stream), "event");
        }
        cuda_ok(cudaStreamSynchronize(g->stream), "draws");
    }
    const int64_t ring = (2 * NX + 2 * (NY - 2)) * NZ;
    ic_ghost_kernel<<<(unsigned)std::min<int64_t>((ring + 255) / 256, (int64_t)g->num_sms * 8), 256, 0, g->stream>>>(
        t, NX, NY, NZ);
    cuda_ok(cudaGetLastError(), "ic_ghost_kernel");
}

// Puts field q, given on the device in the reference layout (contiguous nx*ny*nz FP64, the
// handle's planes), into both state buffers in the handle's own form.
void place_field(r3d_gpu* g, int q, const double* src, const Fp64Staging* stg) {
    const Derived& d = g->d;
    if (g->fp32) {
        to_fp32_kernel<<<stg->blocks(), 256, 0, g->stream>>>(g->X32[0][q], g->geo.pitch, g->geo.plane, src, d.nx,
                                                             d.ny, d.nz, stg->bg(q));
        cuda_ok(cudaGetLastError(), "state32");
        // the second buffer gets the same contents on the device (its z ghost planes are never
        // written by a stage)
        cuda_ok(cudaMemcpyAsync(g->X32[1][q], g->X32[0][q], (size_t)g->geo.plane * d.nz * sizeof(float),
                                cudaMemcpyDeviceToDevice, g->stream),
                "state32");
    } else {
        cuda_ok(cudaMemcpy2DAsync(g->X[0][q], g->geo.pitch * sizeof(double), src, d.nx * sizeof(double),
                                  d.nx * sizeof(double), d.ny * d.nz, cudaMemcpyDeviceToDevice, g->stream),
                "state");
        cuda_ok(cudaMemcpyAsync(g->X[1][q], g->X[0][q], (size_t)g->geo.plane * d.nz * sizeof(double),
                                cudaMemcpyDeviceToDevice, g->stream),
                "state");
    }
}

// The scalars, the dt reduction's start and the dt limits of the new state (end of an upload).
void finish_state(r3d_gpu* g, const r3d_scalars* sc) {
    g->cur = 0;
    r3dk::Scalars h{};
    h.dt = sc->dt; h.timc = sc->timc; h.timt = sc->timt; h.timi = sc->timi;
    h.umach = sc->umach; h.tb = sc->tb; h.nit = sc->nit;
    h.thr_on = g->dt_filter ? 1 : 0;
    h.thr_local = (g->z0 != 0 || g->nloc != g->p.npz) ? 1 : 0;
    h.thr_margin = g->thr_margin;
    *g->hsc = h;
    cuda_ok(cudaMemcpyAsync(g->dsc, g->hsc, sizeof(h), cudaMemcpyHostToDevice, g->stream), "upload scalars");
    g->bnd.tb = sc->tb;
    g->host_timc = sc->timc;
    g->host_timi = sc->timi;
    cuda_ok(r3dk::launch_reset_reduction(g->dsc, g->stream), "reset");
    launch_dt_full_any(g);
    cuda_ok(cudaStreamSynchronize(g->stream), "upload");
    g->uploaded = true;
    g->work_ok = false;
}

}  // namespace r3dg

int r3d_gpu_upload(r3d_gpu* g, const r3d_host_state* st, const r3d_scalars* sc) {
    return guarded([&] {
        if (!g || !st || !sc) throw std::invalid_argument("null argument");
        DeviceGuard dg(g->device);
        Range r("r3d.upload");
        const Derived& d = g->d;
        const double* src[r3dk::kMaxFields] = {st->ru, st->rv, st->rw, st->ro, st->tt, st->bx, st->by, st->bz};
        for (int q = 0; q < g->nfields; ++q)
            if (!src[q]) throw std::invalid_argument("r3d_host_state field is NULL");
        const double* lines[] = {st->dxxdx, st->d2xxdx2, st->ddx, st->exx, st->dyydy, st->d2yydy2,
                                 st->ddy, st->wyy, st->dzzdz, st->d2zzdz2, st->ddz, st->rkapa, st->dkapa};
        for (auto l : lines)
            if (!l) throw std::invalid_argument("r3d_host_state metric line is NULL");
        upload_lines(g, st);
        const size_t n = (size_t)d.nx * d.ny * d.nz;
        if (g->fp32) {
            upload_background(g, st);
            // each field: one contiguous FP64 copy into a staging buffer, then the deviation from
            // the background and the rounding to FP32 on the device
            Fp64Staging stg(g);
            for (int q = 0; q < 5; ++q) {
                cuda_ok(cudaMemcpyAsync(stg.buf, src[q], n * sizeof(double), cudaMemcpyHostToDevice, g->stream),
                        "upload state32");
                place_field(g, q, stg.buf, &stg);
            }
        } else {
            for (int q = 0; q < g->nfields; ++q) {
                // one contiguous host-to-device copy into the accumulator (dead between steps:
                // the first stage rewrites it), then the re-pitch on the device - a pitched
                // host-to-device copy runs at about half the link rate
                cuda_ok(cudaMemcpyAsync(g->Z[q], src[q], n * sizeof(double), cudaMemcpyHostToDevice, g->stream),
                        "upload state");
                place_field(g, q, g->Z[q], nullptr);
            }
        }
        finish_state(g, sc);
    });
}

int r3d_gpu_setup(r3d_gpu* g, r3d_scalars* sc) {
    return guarded([&] {
        if (!g || !sc) throw std::invalid_argument("null argument");
        DeviceGuard dg(g->device);
        Range r("r3d.setup");
        const r3d_params& p = g->p;
        const Derived& d = g->d;
        const int64_t NX = d.nx, NY = d.ny, NZ = d.nz;
        // metric lines and background columns on the host (1D), then uploaded as by r3d_gpu_upload
        std::vector<double> lines[14];
        const int64_t len[14] = {NX, NX, NX, NX, NY, NY, NY, NY, NZ, NZ, NZ, NZ, NZ, NZ};
        for (int q = 0; q < 14; ++q) lines[q].assign((size_t)len[q], 0.0);
        r3d_host_state st{};
        double** lp[14] = {&st.exx, &st.dxxdx, &st.d2xxdx2, &st.ddx, &st.wyy, &st.dyydy, &st.d2yydy2,
                           &st.ddy, &st.zee, &st.dzzdz, &st.d2zzdz2, &st.ddz, &st.rkapa, &st.dkapa};
        for (int q = 0; q < 14; ++q) *lp[q] = lines[q].data();
        setup_lines(p, st, g->z0, g->nloc);
        upload_lines(g, &st);
        std::unique_ptr<Fp64Staging> stg;
        if (g->fp32) {
            upload_background(g, &st);
            stg.reset(new Fp64Staging(g));
        }
        const IcColumns c = ic_columns(p, g->z0, g->nloc);
        DeviceBuffer cols(3 * (size_t)NZ * sizeof(double));
        double* dcol = static_cast<double*>(cols.p);
        std::vector<double> hc(c.t);
        hc.insert(hc.end(), c.r.begin(), c.r.end());
        hc.insert(hc.end(), c.bfac.begin(), c.bfac.end());
        cuda_ok(cudaMemcpyAsync(dcol, hc.data(), hc.size() * sizeof(double), cudaMemcpyHostToDevice, g->stream),
                "setup columns");
        const size_t n = (size_t)NX * NY * NZ;
        const unsigned blocks = (unsigned)std::min<size_t>((n + 255) / 256, (size_t)g->num_sms * 16);
        // fields in the order the temperature needs its draws last: momenta, density, B, then T
        const int order[8] = {0, 1, 2, 3, 5, 6, 7, 4};
        for (int oi = 0; oi < 8; ++oi) {
            const int q = order[oi];
            if (q >= g->nfields) continue;
            double* buf = g->fp32 ? stg->buf : g->Z[q];
            const int kind = q == 4 ? 1 : (q == 3 ? 2 : (q == 5 ? 3 : 0));
            ic_field_kernel<<<blocks, 256, 0, g->stream>>>(buf, NX, NY, NZ, kind, dcol, dcol + NZ, dcol + 2 * NZ,
                                                          d.obeta, p.lmag, g->z0, (int64_t)p.npz + 2);
            cuda_ok(cudaGetLastError(), "ic_field_kernel");
            if (q == 4) perturb_temperature(g, buf);
            place_field(g, q, buf, stg.get());
        }
        r3d_scalars s{};
        s.tb = c.tb;
        finish_state(g, &s);
        *sc = s;
    });
}

int r3d_gpu_download(r3d_gpu* g, r3d_host_state* st, r3d_scalars* sc) {
    return guarded([&] {
        if (!g || !st) throw std::invalid_argument("null argument");
        if (!g->uploaded) throw Error(R3D_ESTATE, "download before upload");
        DeviceGuard dg(g->device);
        Range r("r3d.download");
        const Derived& d = g->d;
        double* dst[r3dk::kMaxFields] = {st->ru, st->rv, st->rw, st->ro, st->tt, st->bx, st->by, st->bz};
        if (g->fp32) {
            Fp64Staging stg(g);
            for (int q = 0; q < 5; ++q) {
                if (!dst[q]) continue;
                from_fp32_kernel<<<stg.blocks(), 256, 0, g->stream>>>(stg.buf, g->X32[g->cur][q], g->geo.pitch,
                                                                      g->geo.plane, d.nx, d.ny, d.nz, stg.bg(q));
                cuda_ok(cudaGetLastError(), "download state32");
                cuda_ok(cudaMemcpyAsync(dst[q], stg.buf, stg.n * sizeof(double), cudaMemcpyDeviceToHost, g->stream),
                        "download state32");
            }
            cuda_ok(cudaStreamSynchronize(g->stream), "download state32");
        } else {
            for (int q = 0; q < g->nfields; ++q) {
                if (!dst[q]) continue;
                cuda_ok(cudaMemcpy2DAsync(dst[q], d.nx * sizeof(double), g->X[g->cur][q],
                                          g->geo.pitch * sizeof(double), d.nx * sizeof(double), d.ny * d.nz,
                                          cudaMemcpyDeviceToHost, g->stream),
                        "download state");
            }
        }
        pull_scalars(g, sc);
    });
}

int r3d_gpu_download_accumulators(r3d_gpu* g, double* const* z) {
    return guarded([&] {
        if (!g || !z) throw std::invalid_argument("null argument");
        if (!g->uploaded) throw Error(R3D_ESTATE, "download before upload");
        DeviceGuard dg(g->device);
        Range r("r3d.download");
        const Derived& d = g->d;
        if (g->fp32) {
            Fp64Staging stg(g);
            for (int q = 0; q < 5; ++q) {
                if (!z[q]) continue;
                z_from_fp32_kernel<<<stg.blocks(), 256, 0, g->stream>>>(stg.buf, g->Z32[q], g->geo.pitch, g->geo.plane,
                                                                        d.nx, d.ny, d.nz, stg.bg(q));
                cuda_ok(cudaGetLastError(), "download accumulators32");
                cuda_ok(cudaMemcpyAsync(z[q], stg.buf, stg.n * sizeof(double), cudaMemcpyDeviceToHost, g->stream),
                        "download accumulators32");
            }
        } else {
            for (int q = 0; q < g->nfields; ++q) {
                if (!z[q]) continue;
                cuda_ok(cudaMemcpy2DAsync(z[q], d.nx * sizeof(double), g->Z[q], g->geo.pitch * sizeof(double),
                                          d.nx * sizeof(double), d.ny * d.nz, cudaMemcpyDeviceToHost, g->stream),
                        "download accumulators");
            }
        }
        cuda_ok(cudaStreamSynchronize(g->stream), "download accumulators");
    });
}

namespace r3dg {

// FLUXES of the FP64 state in buffer set `buf` (without changing it) into host arrays out[0 ..
// nfields-1] (NX*NY*NZ each, interior cells, ghosts 0); null entries are skipped.  The stage
// kernel runs as a first stage with its F stored, into scratch kept by the handle.
void eval_fluxes(r3d_gpu* g, int buf, double* const* out) {
    const Derived& d = g->d;
    const size_t fe = (size_t)g->geo.plane * d.nz;
    const int nf = g->nfields;
    if (!g->fscr) {
        cuda_ok(cudaMalloc(&g->fscr, 3 * (size_t)nf * fe * sizeof(double)), "cudaMalloc(flux scratch)");
        cuda_ok(cudaMemsetAsync(g->fscr, 0, 3 * (size_t)nf * fe * sizeof(double), g->stream), "cudaMemset");
        g->bytes += (int64_t)(3 * (size_t)nf * fe * sizeof(double));
    }
    FieldSet fs{};
    for (int q = 0; q < nf; ++q) {
        fs.xin[q] = g->X[buf][q];
        fs.xout[q] = g->fscr + (size_t)q * fe;                 // stage result, discarded
        fs.z[q] = g->fscr + (size_t)(nf + q) * fe;             // accumulator, discarded
        fs.f[q] = g->fscr + (size_t)(2 * nf + q) * fe;         // F
    }
    cuda_ok(r3dk::launch_stage_fp64(0, g->maps[buf], g->geo, g->ph, g->lines, fs, g->dsc, g->kchunk, g->stream,
                                    true),
            "fluxes");
    std::vector<double> hb((size_t)(d.nx * d.ny * d.nz));
    for (int q = 0; q < nf; ++q) {
        if (!out[q]) continue;
        cuda_ok(cudaMemcpy2DAsync(hb.data(), d.nx * sizeof(double), fs.f[q], g->geo.pitch * sizeof(double),
                                  d.nx * sizeof(double), d.ny * d.nz, cudaMemcpyDeviceToHost, g->stream),
                "fluxes download");
        cuda_ok(cudaStreamSynchronize(g->stream), "fluxes");
        for (int64_t k = 0; k < d.nz; ++k)
            for (int64_t j = 0; j < d.ny; ++j)
                for (int64_t i = 0; i < d.nx; ++i) {
                    const bool inner = k >= 1 && k <= d.nz - 2 && j >= 1 && j <= d.ny - 2 && i >= 1 && i <= d.nx - 2;
                    const size_t n = (size_t)((k * d.ny + j) * d.nx + i);
                    out[q][n] = inner ? hb[n] : 0.0;
                }
    }
}

}  // namespace r3dg

int r3d_gpu_fluxes(r3d_gpu* g, double* const* out) {
    return guarded([&] {
        if (!g || !out) throw std::invalid_argument("null argument");
        if (!g->uploaded) throw Error(R3D_ESTATE, "fluxes before upload");
        if (g->fp32) throw Error(R3D_EINVAL, "r3d_gpu_fluxes needs precision fp64");
        if (g->p.id != 0) throw Error(R3D_EINVAL, "r3d_gpu_fluxes does not form the density diffusion (ID)");
        DeviceGuard dg(g->device);
        for (int q = 0; q < g->nfields; ++q)
            if (!out[q]) throw std::invalid_argument("null output field");
        eval_fluxes(g, g->cur, out);
        pull_scalars(g, nullptr);
    });
}

int r3d_gpu_download_work(r3d_gpu* g, double* const* out) {
    return guarded([&] {
        if (!g || !out) throw std::invalid_argument("null argument");
        if (!g->uploaded) throw Error(R3D_ESTATE, "download before upload");
        if (g->fp32) throw Error(R3D_EINVAL, "r3d_gpu_download_work needs precision fp64");
        if (!g->work_ok) throw Error(R3D_ESTATE, "no full step since the state was set");
        bool want_f = false;
        for (int q = 3; q < 8; ++q) want_f = want_f || out[q];
        if (want_f && g->p.id != 0)
            throw Error(R3D_EINVAL, "the fluxes with density diffusion (ID) are not formed outside a stage");
        DeviceGuard dg(g->device);
        const Derived& d = g->d;
        const int prev = 1 - g->cur;  // after a full step: the third stage's input
        const size_t cnt = (size_t)(d.nx * d.ny * d.nz);
        if (out[0] || out[1] || out[2]) {
            // UU = RU * (1/RO) etc. over the whole local array (src/fluxes.cpp:131-165)
            std::vector<double> h(4 * cnt);
            for (int q = 0; q < 4; ++q)
                cuda_ok(cudaMemcpy2DAsync(h.data() + q * cnt, d.nx * sizeof(double), g->X[prev][q],
                                          g->geo.pitch * sizeof(double), d.nx * sizeof(double), d.ny * d.nz,
                                          cudaMemcpyDeviceToHost, g->stream),
                        "download work");
            cuda_ok(cudaStreamSynchronize(g->stream), "download work");
            for (size_t n = 0; n < cnt; ++n) {
                const double rinv = 1.0 / h[3 * cnt + n];
                for (int q = 0; q < 3; ++q)
                    if (out[q]) out[q][n] = h[q * cnt + n] * rinv;
            }
        }
        if (want_f) {
            double* fo[r3dk::kMaxFields] = {};
            for (int q = 0; q < 5; ++q) fo[q] = out[3 + q];
            eval_fluxes(g, prev, fo);
        }
    });
}

int r3d_gpu_debug_tma_extra(r3d_gpu* g, unsigned int bytes) {
    return guarded([&] {
        if (!g) throw std::invalid_argument("null handle");
        DeviceGuard dg(g->device);
        cuda_ok(cudaMemcpyAsync(&g->dsc->tx_extra, &bytes, sizeof bytes, cudaMemcpyHostToDevice, g->stream),
                "tx_extra");
        cuda_ok(cudaStreamSynchronize(g->stream), "tx_extra");
    });
}

int r3d_gpu_debug_dt_filter(r3d_gpu* g, double margin, int* refolds) {
    return guarded([&] {
        if (!g) throw std::invalid_argument("null handle");
        DeviceGuard dg(g->device);
        if (!std::isnan(margin)) {
            g->thr_margin = margin;
            cuda_ok(cudaMemcpyAsync(&g->dsc->thr_margin, &g->thr_margin, sizeof(double), cudaMemcpyHostToDevice,
                                    g->stream),
                    "thr_margin");
        }
        if (refolds) {
            cuda_ok(cudaMemcpyAsync(&g->hsc->refolds, &g->dsc->refolds, sizeof(int), cudaMemcpyDeviceToHost,
                                    g->stream),
                    "refolds");
        }
        cuda_ok(cudaStreamSynchronize(g->stream), "dt filter");
        if (refolds) *refolds = g->hsc->refolds;
    });
}

int r3d_gpu_memory(const r3d_gpu* g, int64_t* bytes) {
    if (!g || !bytes) return R3D_EINVAL;
    *bytes = g->bytes;
    return R3D_OK;
}

void* r3d_gpu_stream(r3d_gpu* g) { return g ? (void*)g->stream : nullptr; }

int r3d_gpu_plan(const r3d_params* p, int nloc, int num_sms, int* kchunk, int* tile_rows) {
    return guarded([&] {
        if (!p || !kchunk || !tile_rows) throw std::invalid_argument("r3d_gpu_plan: null argument");
        check_params(*p);
        const int n = nloc > 0 ? nloc : p->npz;
        if (n < 4 || n > p->npz) throw std::invalid_argument("r3d_gpu_plan: nloc must lie in [4, npz]");
        int sms = num_sms;
        if (sms <= 0) {
            DeviceGuard dg(p->gpu_id);
            cuda_ok(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, p->gpu_id),
                    "cudaDeviceGetAttribute(multiprocessors)");
        }
        const bool fp32 = p->precision == R3D_PREC_FP32BULK;
        const int rows = r3dk::stage_fp64_rows(p->lmag, p->npx, p->npy, n, sms);
        unsigned bx = 0, by = 0;
        if (fp32) r3dk::stage_fp32_box(&bx, &by);
        else r3dk::stage_fp64_box(rows, &bx, &by);
        *tile_rows = (int)by - 2;
        *kchunk = stage_chunk_depth(*p, fp32, rows, n, sms);
    });
}

int r3d_gpu_step(r3d_gpu* g, int nstages, r3d_scalars* sc) {
    return guarded([&] {
        if (!g) throw std::invalid_argument("null handle");
        if (nstages < 1 || nstages > 3) throw std::invalid_argument("nstages must be 1..3");
        if (!g->uploaded) throw Error(R3D_ESTATE, "step before upload");
        DeviceGuard dg(g->device);
        Timer tm{g, false, nullptr};
        int a = 0, b = 0;
        enqueue_step(g, nstages, tm, a, b);
        r3d_scalars tmp{};
        pull_scalars(g, &tmp);
        if (sc) *sc = tmp;
        if (!std::isfinite(tmp.dt)) throw Error(R3D_ENUMERIC, "non-finite dt");
    });
}

int r3d_gpu_run(r3d_gpu* g, int nsteps, r3d_scalars* sc) {
    return guarded([&] { run_steps(g, nsteps, sc, nullptr, true); });
}

int r3d_gpu_enqueue(r3d_gpu* g, int nsteps) {
    return guarded([&] { run_steps(g, nsteps, nullptr, nullptr, false); });
}

int r3d_gpu_run_timed(r3d_gpu* g, int nsteps, r3d_scalars* sc, r3d_timing* tm) {
    return guarded([&] {
        if (!tm) throw std::invalid_argument("null timing");
        run_steps(g, nsteps, sc, tm, true);
    });
}

int r3d_gpu_totals(r3d_gpu* g, double* mass, double* energy) {
    return guarded([&] {
        if (!g || !g->uploaded) throw Error(R3D_ESTATE, "totals before upload");
        DeviceGuard dg(g->device);
        double zero[2] = {0.0, 0.0};
        cuda_ok(cudaMemcpyAsync(&g->dsc->mass, zero, sizeof(zero), cudaMemcpyHostToDevice, g->stream), "totals");
        if (g->fp32)
            cuda_ok(r3dk::launch_totals_fp32(g->geo, g->ph, g->bg, fieldset32(g), g->dsc, g->stream), "totals32");
        else
            cuda_ok(r3dk::launch_totals(g->geo, g->ph, fieldset(g), g->dsc, g->stream), "totals");
        cuda_ok(cudaMemcpyAsync(zero, &g->dsc->mass, sizeof(zero), cudaMemcpyDeviceToHost, g->stream), "totals");
        cuda_ok(cudaStreamSynchronize(g->stream), "totals");
        if (mass) *mass = zero[0];
        if (energy) *energy = zero[1];
    });
}

}  // extern "C"
