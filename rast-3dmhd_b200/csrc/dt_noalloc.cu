// dt_noalloc.cu - time-step limits of a caller-owned device state, allocating nothing.
//
// Who needs this: callers that cannot call cudaMalloc.  Typical cases are a host program that
// reserves the GPU's memory up front in its own pool for the simulation fields and lets no
// library allocate beside it, and a time loop that must not pay the device synchronisation
// that cudaMalloc/cudaFree may imply.  The regular path keeps its reduction accumulators in
// memory allocated by r3d_gpu_create; this entry point instead keeps the per-block partial
// results in one file-scope __device__ array (g_dt_partials below), which every GPU that loads
// the library holds until the process exits.
//
// Limits and sharing:
//  * at most kMaxBlocks partial slots: one per 32 x 8 column tile, so npx*npy is limited to
//    ceil(npx/32) * ceil(npy/8) <= 65536 tiles (2.5 MiB of partials), and ceil(npy/8) to the
//    65535 blocks a launch may have along y; larger grids are rejected with R3D_EINVAL before
//    anything runs;
//  * every call on a device uses the same array, and the array keeps the last call's partials;
//    nothing in it has to start at zero (pass 1 writes every slot pass 2 reads), but two calls
//    whose kernels overlap on the GPU (different streams, no ordering) race on the array;
//  * every call looks up the array's device address with cudaGetSymbolAddress, with the
//    target device current.  The first lookup in a CUDA context loads this module onto the
//    device, so make the first call on a device before any stream capture; later lookups are
//    host-side and cheap.  Nothing is cached across calls, so a cudaDeviceReset (which may
//    reload the module at another address) needs no special handling.
#include <cuda_runtime.h>

#include <string>

#include "r3d_device.cuh"
#include "r3d_error.hpp"
#include "r3d_gpu.h"
#include "r3d_host.hpp"
#include "stage_common.cuh"

namespace {

constexpr int kTileX = 32, kTileY = 8;
constexpr int kMaxBlocks = 65536;

// Per-tile partial limits: min ww1, min ww2, min ww3, min vv, max Mach term.
static __device__ __align__(256) double g_dt_partials[5 * kMaxBlocks];


struct Inputs {
    const double* f[8];  // ru rv rw ro tt bx by bz (reference layout, x fastest)
    const double *ddx, *ddy, *ddz, *rkapa;
    int64_t nx, ny;
};

// Pass 1: one block per column tile folds its cells (every k) into one partial slot.
__global__ void __launch_bounds__(kTileX* kTileY) dt_partials_kernel(r3dk::Physics ph, int npx,
                                                                     int npy, int npz, Inputs in,
                                                                     double* partials) {
    __shared__ double red[5 * 8];
    const int i = 1 + blockIdx.x * kTileX + threadIdx.x;
    const int j = 1 + blockIdx.y * kTileY + threadIdx.y;
    double m1 = 1e300, m2 = 1e300, m3 = 1e300, m4 = 1e300, mu = 0.0;
    if (i <= npx && j <= npy) {
        const double dxy = (in.ddy[j] < in.ddx[i]) ? in.ddy[j] : in.ddx[i];
        for (int k = 1; k <= npz; ++k) {
            const int64_t n = ((int64_t)k * in.ny + j) * in.nx + i;
            double b2 = 0.0;
            if (ph.lmag) {
                const double bx = in.f[5][n], by = in.f[6][n], bz = in.f[7][n];
                b2 = bx * bx + by * by + bz * bz;
            }
            const double dd = (in.ddz[k] < dxy) ? in.ddz[k] : dxy;
            double w1, w2, w3, w4, um;
            r3dk::dt_terms(ph, in.f[0][n], in.f[1][n], in.f[2][n], in.f[3][n], in.f[4][n], b2, dd,
                           in.rkapa[k], w1, w2, w3, w4, um);
            m1 = r3dk::fold_min(m1, w1);
            m2 = r3dk::fold_min(m2, w2);
            m3 = r3dk::fold_min(m3, w3);
            m4 = r3dk::fold_min(m4, w4);
            mu = r3dk::fold_max(mu, um);
        }
    }
    // block fold (warp shuffles, then one row of the block)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        m1 = r3dk::fold_min(m1, __shfl_xor_sync(0xffffffffu, m1, o));
        m2 = r3dk::fold_min(m2, __shfl_xor_sync(0xffffffffu, m2, o));
        m3 = r3dk::fold_min(m3, __shfl_xor_sync(0xffffffffu, m3, o));
        m4 = r3dk::fold_min(m4, __shfl_xor_sync(0xffffffffu, m4, o));
        mu = r3dk::fold_max(mu, __shfl_xor_sync(0xffffffffu, mu, o));
    }
    const int tid = threadIdx.y * kTileX + threadIdx.x;
    if ((tid & 31) == 0) {
        const int w = tid >> 5;
        red[w * 5 + 0] = m1;
        red[w * 5 + 1] = m2;
        red[w * 5 + 2] = m3;
        red[w * 5 + 3] = m4;
        red[w * 5 + 4] = mu;
    }
    __syncthreads();
    if (tid == 0) {
        for (int w = 1; w < 8; ++w) {
            m1 = r3dk::fold_min(m1, red[w * 5 + 0]);
            m2 = r3dk::fold_min(m2, red[w * 5 + 1]);
            m3 = r3dk::fold_min(m3, red[w * 5 + 2]);
            m4 = r3dk::fold_min(m4, red[w * 5 + 3]);
            mu = r3dk::fold_max(mu, red[w * 5 + 4]);
        }
        double* slot = partials + 5 * (int64_t)(blockIdx.y * gridDim.x + blockIdx.x);
        slot[0] = m1;
        slot[1] = m2;
        slot[2] = m3;
        slot[3] = m4;
        slot[4] = mu;
    }
}

// Pass 2: one block folds the nblocks partials; out = {dt, umach} (src/step.cpp:141,224-229).
__global__ void __launch_bounds__(256) dt_final_kernel(r3dk::Physics ph, const double* partials,
                                                       int nblocks, double* out) {
    __shared__ double red[5 * 8];
    double m1 = 1e300, m2 = 1e300, m3 = 1e300, m4 = 1e300, mu = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
        const double* s = partials + 5 * (int64_t)b;
        m1 = r3dk::fold_min(m1, s[0]);
        m2 = r3dk::fold_min(m2, s[1]);
        m3 = r3dk::fold_min(m3, s[2]);
        m4 = r3dk::fold_min(m4, s[3]);
        mu = r3dk::fold_max(mu, s[4]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        m1 = r3dk::fold_min(m1, __shfl_xor_sync(0xffffffffu, m1, o));
        m2 = r3dk::fold_min(m2, __shfl_xor_sync(0xffffffffu, m2, o));
        m3 = r3dk::fold_min(m3, __shfl_xor_sync(0xffffffffu, m3, o));
        m4 = r3dk::fold_min(m4, __shfl_xor_sync(0xffffffffu, m4, o));
        mu = r3dk::fold_max(mu, __shfl_xor_sync(0xffffffffu, mu, o));
    }
    if ((threadIdx.x & 31) == 0) {
        const int w = threadIdx.x >> 5;
        red[w * 5 + 0] = m1;
        red[w * 5 + 1] = m2;
        red[w * 5 + 2] = m3;
        red[w * 5 + 3] = m4;
        red[w * 5 + 4] = mu;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < 8; ++w) {
            m1 = r3dk::fold_min(m1, red[w * 5 + 0]);
            m2 = r3dk::fold_min(m2, red[w * 5 + 1]);
            m3 = r3dk::fold_min(m3, red[w * 5 + 2]);
            m4 = r3dk::fold_min(m4, red[w * 5 + 3]);
            mu = r3dk::fold_max(mu, red[w * 5 + 4]);
        }
        double m = (m2 < m1) ? m2 : m1;
        m = (m3 < m) ? m3 : m;
        if (ph.lmag) m = (m4 < m) ? m4 : m;
        out[0] = ph.sff * m;
        out[1] = sqrt(mu);
    }
}

// Device address of g_dt_partials in the current context (the target device is current).  Host
// code holds only a host-side stand-in under the array's name; the kernels need this address.
double* partials_address() {
    void* ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_dt_partials);
    if (e != cudaSuccess || !ptr)
        throw r3db::Error(R3D_ECUDA, std::string("cudaGetSymbolAddress(g_dt_partials): ") +
                                         cudaGetErrorString(e));
    return static_cast<double*>(ptr);
}

}  // namespace

extern "C" int r3d_dt_limits_noalloc(const r3d_params* p, const double* const* fields,
                                     const double* const* lines, double* out, void* stream) {
    using namespace r3db;
    return guarded([&] {
        if (!p || !fields || !lines || !out) throw std::invalid_argument("null argument");
        check_params(*p);
        const int nf = p->lmag ? 8 : 5;
        Inputs in{};
        for (int q = 0; q < nf; ++q) {
            if (!fields[q]) throw std::invalid_argument("field pointer is NULL");
            in.f[q] = fields[q];
        }
        for (int q = 0; q < 4; ++q)
            if (!lines[q]) throw std::invalid_argument("metric line pointer is NULL");
        in.ddx = lines[0];
        in.ddy = lines[1];
        in.ddz = lines[2];
        in.rkapa = lines[3];
        in.nx = (int64_t)p->npx + 2;
        in.ny = (int64_t)p->npy + 2;
        const int64_t bx = (p->npx + kTileX - 1) / kTileX, by = (p->npy + kTileY - 1) / kTileY;
        if (bx * by > kMaxBlocks)
            throw std::invalid_argument("grid too large for r3d_dt_limits_noalloc: " +
                                        std::to_string(bx * by) + " column tiles of 32x8, the fixed "
                                        "partials array holds " + std::to_string(kMaxBlocks));
        if (by > 65535)
            throw std::invalid_argument("grid too large for r3d_dt_limits_noalloc: npy = " +
                                        std::to_string(p->npy) + " needs " + std::to_string(by) +
                                        " tile rows, a launch holds at most 65535");
        if (p->gpu_id < 0) throw std::invalid_argument("gpu id out of range");
        int prev = -1;
        cudaGetDevice(&prev);
        if (prev != p->gpu_id) {
            const cudaError_t e = cudaSetDevice(p->gpu_id);
            if (e != cudaSuccess) throw Error(R3D_ECUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
        }
        struct Restore {
            int dev;
            ~Restore() {
                if (dev >= 0) cudaSetDevice(dev);
            }
        } restore{prev != p->gpu_id ? prev : -1};
        double* partials = partials_address();
        const Derived d = derive(*p);
        r3dk::Physics ph{};
        ph.gamma = p->gamma;
        ph.ogamma = 1.0 / p->gamma;
        ph.re = p->re;
        ph.repr = d.repr;
        ph.cv = d.cv;
        ph.rm = p->rm;
        ph.obeta = d.obeta;
        ph.sff = p->sf;
        ph.lmag = p->lmag;
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        dt_partials_kernel<<<dim3((unsigned)bx, (unsigned)by, 1), dim3(kTileX, kTileY, 1), 0, st>>>(
            ph, p->npx, p->npy, p->npz, in, partials);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) {
            dt_final_kernel<<<1, 256, 0, st>>>(ph, partials, (int)(bx * by), out);
            e = cudaGetLastError();
        }
        if (e != cudaSuccess) throw Error(R3D_ECUDA, std::string("dt_noalloc launch: ") + cudaGetErrorString(e));
    });
}
