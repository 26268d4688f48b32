// compare.cu - error norms between two device states of the same grid, on the device.
//
// r3d_gpu_compare(a, ref, out): for every field of ref (ru rv rw ro tt [bx by bz]) the sums
// sum (a - ref)^2, sum ref^2 and the maxima max |a - ref|, max |ref| over the interior cells.
// Either handle may hold the FP64 form or the FP32-bulk form; the latter's rho and T are
// compared as full values, background column + deviation (the form its download produces).
// This is how the FP32-bulk error is measured on grids whose two host copies would not fit
// in host memory (504 x 504 x 2048: 2 x 21 GB).
//
// Deterministic: each block writes its partial sums to its own slot and the host adds the
// slots in block order, so the same states give the same bits on every call.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "r3d_device.cuh"
#include "r3d_error.hpp"
#include "r3d_gpu.h"
#include "r3d_gpu_impl.hpp"
#include "r3d_kernels.h"

namespace {

constexpr int kTx = 32, kTy = 8, kMaxZ = 64;

// One state as the comparison reads it: FP64 arrays, or FP32 arrays plus the background
// columns of rho and T (indexed by the local plane).
struct Src {
    const double* d[r3dk::kMaxFields];
    const float* f[r3dk::kMaxFields];
    const double* bg_r;
    const double* bg_t;
    int64_t pitch, plane;
};

__device__ __forceinline__ double value(const Src& s, int q, int i, int j, int k) {
    const int64_t n = (int64_t)k * s.plane + (int64_t)j * s.pitch + i;
    if (s.f[q]) {
        const double b = q == 3 ? s.bg_r[k] : (q == 4 ? s.bg_t[k] : 0.0);
        return b + (double)s.f[q][n];
    }
    return s.d[q][n];
}

// partials[block][q][4] = {sum d^2, sum r^2, max |d|, max |r|}
__global__ void __launch_bounds__(kTx* kTy) compare_kernel(int npx, int npy, int npz, int nf, Src a, Src r,
                                                           double* partials) {
    __shared__ double red[kTx * kTy / 32][r3dk::kMaxFields][4];
    const int i = 1 + blockIdx.x * kTx + threadIdx.x;
    const int j = 1 + blockIdx.y * kTy + threadIdx.y;
    double acc[r3dk::kMaxFields][4];
#pragma unroll
    for (int q = 0; q < r3dk::kMaxFields; ++q) acc[q][0] = acc[q][1] = acc[q][2] = acc[q][3] = 0.0;
    if (i <= npx && j <= npy) {
        for (int k = 1 + blockIdx.z; k <= npz; k += gridDim.z) {
#pragma unroll
            for (int q = 0; q < r3dk::kMaxFields; ++q) {
                if (q >= nf) break;
                const double rv = value(r, q, i, j, k);
                const double d = value(a, q, i, j, k) - rv;
                acc[q][0] += d * d;
                acc[q][1] += rv * rv;
                acc[q][2] = fmax(acc[q][2], fabs(d));
                acc[q][3] = fmax(acc[q][3], fabs(rv));
            }
        }
    }
    const int tid = threadIdx.y * kTx + threadIdx.x, w = tid >> 5;
#pragma unroll
    for (int q = 0; q < r3dk::kMaxFields; ++q) {
        if (q >= nf) break;
        for (int o = 16; o > 0; o >>= 1) {
            acc[q][0] += __shfl_xor_sync(0xffffffffu, acc[q][0], o);
            acc[q][1] += __shfl_xor_sync(0xffffffffu, acc[q][1], o);
            acc[q][2] = fmax(acc[q][2], __shfl_xor_sync(0xffffffffu, acc[q][2], o));
            acc[q][3] = fmax(acc[q][3], __shfl_xor_sync(0xffffffffu, acc[q][3], o));
        }
        if ((tid & 31) == 0)
            for (int s = 0; s < 4; ++s) red[w][q][s] = acc[q][s];
    }
    __syncthreads();
    if (tid < nf * 4) {
        const int q = tid / 4, s = tid % 4;
        double v = red[0][q][s];
        for (int ww = 1; ww < kTx * kTy / 32; ++ww) v = s < 2 ? v + red[ww][q][s] : fmax(v, red[ww][q][s]);
        const int64_t b = ((int64_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
        partials[(b * nf + q) * 4 + s] = v;
    }
}

Src source(const r3d_gpu* g) {
    Src s{};
    for (int q = 0; q < g->nfields; ++q) {
        if (g->fp32) s.f[q] = g->X32[g->cur][q];
        else s.d[q] = g->X[g->cur][q];
    }
    s.bg_r = g->bg.r;
    s.bg_t = g->bg.t;
    s.pitch = g->geo.pitch;
    s.plane = g->geo.plane;
    return s;
}

}  // namespace

extern "C" int r3d_gpu_compare(const r3d_gpu* a, const r3d_gpu* ref, double* out) {
    using namespace r3db;
    return guarded([&] {
        if (!a || !ref || !out) throw std::invalid_argument("r3d_gpu_compare: null argument");
        if (!a->uploaded || !ref->uploaded) throw Error(R3D_ESTATE, "compare before upload");
        if (a->p.npx != ref->p.npx || a->p.npy != ref->p.npy || a->p.npz != ref->p.npz || a->z0 != ref->z0 ||
            a->nloc != ref->nloc || a->nfields != ref->nfields)
            throw std::invalid_argument("r3d_gpu_compare: the two handles hold different grids or fields");
        if (a->device != ref->device) throw std::invalid_argument("r3d_gpu_compare: handles on different devices");
        r3dg::DeviceGuard dg(ref->device);
        const int nf = ref->nfields;
        const dim3 block(kTx, kTy, 1);
        const dim3 grid((a->geo.npx + kTx - 1) / kTx, (a->geo.npy + kTy - 1) / kTy,
                        (unsigned)std::min(a->geo.npz, kMaxZ));
        const size_t nblocks = (size_t)grid.x * grid.y * grid.z;
        const size_t nval = nblocks * nf * 4;
        double* dpart = nullptr;
        r3dg::cuda_ok(cudaMalloc(&dpart, nval * sizeof(double)), "cudaMalloc(compare partials)");
        struct Free {
            double* p;
            ~Free() { cudaFree(p); }
        } free_partials{dpart};
        // both states are final once the reference handle's stream and the other's have drained
        r3dg::cuda_ok(cudaStreamSynchronize(a->stream), "compare: drain");
        compare_kernel<<<grid, block, 0, ref->stream>>>(a->geo.npx, a->geo.npy, a->geo.npz, nf, source(a),
                                                         source(ref), dpart);
        r3dg::cuda_ok(cudaGetLastError(), "compare_kernel launch");
        std::vector<double> part(nval);
        r3dg::cuda_ok(cudaMemcpyAsync(part.data(), dpart, nval * sizeof(double), cudaMemcpyDeviceToHost, ref->stream),
                "compare: partials");
        r3dg::cuda_ok(cudaStreamSynchronize(ref->stream), "compare");
        for (int q = 0; q < nf; ++q) out[4 * q] = out[4 * q + 1] = out[4 * q + 2] = out[4 * q + 3] = 0.0;
        for (size_t b = 0; b < nblocks; ++b)
            for (int q = 0; q < nf; ++q) {
                const double* v = &part[(b * nf + q) * 4];
                out[4 * q] += v[0];
                out[4 * q + 1] += v[1];
                out[4 * q + 2] = std::max(out[4 * q + 2], v[2]);
                out[4 * q + 3] = std::max(out[4 * q + 3], v[3]);
            }
    });
}
