// adjoint.cu - discrete adjoint (reverse mode) of the FP64 RK3 step, with checkpointing.
//
// The reference has no adjoint; this is the derivative of exactly the map the forward kernels
// compute (src/step.cpp:114-257 with FLUXES, BCON and the dt reduction).  A trajectory of N
// steps is recorded by the ordinary forward path, keeping the state every K steps on the
// device.  The backward sweep walks the segments in reverse: it recomputes the states of a
// segment from its checkpoint, then for each step (last first) recomputes the three stages
// once more - now also storing the right-hand sides F_s (stage kernels with EMIT) - and runs
//
//   for s = 2, 1, 0:   lambda_Y   = BCON^T lambda_X_{s+1}            (adj_bcon_kernel)
//                      lambda_F_s += gam_s dt lambda_Y               (adj_seed_kernel)
//                      lambda_X_s  = F'(X_s)^T lambda_F_s + lambda_Y (adj_pass1/pass2_kernel)
//                      lambda_F_{s-1} = zeta_s dt lambda_Y
//   lambda_dt = sum_s gam_s <F_s, lambda_Y> + zeta_s <F_{s-1}, lambda_Y>   (deterministic sum)
//   lambda_X_0 += lambda_dt * sff * d(limit)/dX at the cell that set dt (adj_argmin, adj_dt)
//
// Each recomputed step is compared bit for bit with the recorded state that follows it; a
// mismatch (a non-reproducible forward) is reported as R3D_ENUMERIC instead of a silently wrong
// gradient.  Limits: FP64 only; a time-independent top boundary (tc == 0), since the plume
// relaxation clock would otherwise couple every step to the sum of all earlier dt.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "adjoint_cell.cuh"
#include "r3d_gpu_impl.hpp"
#include "stage_common.cuh"

using namespace r3db;
using r3dk::AdjArgs;

namespace {

constexpr int kDots = 5;  // gam_2, gam_1, gam_0 dots (seed) and zeta_2, zeta_1 dots (pass 2)
constexpr int BX = 32, BY = 4;

struct AdjScalars {
    unsigned long long wkey[4];  // the step's four limit minima (ordered keys), saved before dt
    unsigned long long argmin;   // smallest cell index holding the winning limit
    unsigned long long mismatch; // recompute vs recorded state: differing values
    double lam_dt;
    double mstar;
    int term;
};

__device__ __forceinline__ int block_linear() {
    return blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
}

// Deterministic block sum of v (all threads call); thread 0 stores it to out[block].
__device__ void block_sum_store(double v, double* out) {
    __shared__ double red[BX * BY / 32];
    const int tid = threadIdx.x + blockDim.x * threadIdx.y;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((tid & 31) == 0) red[tid >> 5] = v;
    __syncthreads();
    if (tid == 0) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x * blockDim.y) / 32; ++w) s += red[w];
        out[block_linear()] = s;
    }
}

__global__ void __launch_bounds__(BX* BY) adj_bcon_kernel(r3dk::Geometry g, r3dk::Physics ph,
                                                           r3dk::Boundary bd, AdjArgs A) {
    const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
    if (i > g.npx || j > g.npy) return;
    r3dk::adj_bcon_column(g, ph, bd, A.x, A.lam, A.nf, i, j);
}

// lambda_F (+)= gam dt lambda_Y on the interior; partial dot <F_s, lambda_Y> per block.
__global__ void __launch_bounds__(BX* BY) adj_seed_kernel(AdjArgs A, double* lamF0, double* lamF1, double* lamF2,
                                                           double* lamF3, double* lamF4, double* lamF5,
                                                           double* lamF6, double* lamF7, double gam, int first,
                                                           double* dots) {
    const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
    const int k = 1 + blockIdx.z;
    double* lf[8] = {lamF0, lamF1, lamF2, lamF3, lamF4, lamF5, lamF6, lamF7};
    double dot = 0.0;
    if (i <= A.g.npx && j <= A.g.npy) {
        const int n = k * (int)A.g.plane + j * (int)A.g.pitch + i;
        const double gdt = gam * A.sc->dt;
#pragma unroll
        for (int f = 0; f < 8; ++f) {  // unrolled: the pointer table stays in registers
            if (f < A.nf) {
                const double ly = A.lam[f][n];
                lf[f][n] = (first ? 0.0 : lf[f][n]) + gdt * ly;
                dot += A.fprev[f][n] * ly;  // fprev carries F_s here
            }
        }
    }
    block_sum_store(dot, dots);
}

__global__ void __launch_bounds__(BX* BY) adj_pass1_kernel(AdjArgs A) {
    const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
    const int k = 1 + blockIdx.z;
    if (i <= A.g.npx && j <= A.g.npy) r3dk::adj_pass1_cell(A, i, j, k);
}

__global__ void __launch_bounds__(BX* BY) adj_pass2_kernel(AdjArgs A, double* dots) {
    const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
    const int k = 1 + blockIdx.z;
    double dot = 0.0;
    if (i <= A.g.npx && j <= A.g.npy) dot = r3dk::adj_pass2_cell(A, i, j, k);
    if (dots) block_sum_store(dot, dots);
}

__global__ void adj_save_limits_kernel(const r3dk::Scalars* sc, AdjScalars* aux) {
    for (int q = 0; q < 4; ++q) aux->wkey[q] = sc->wmin[q];
}

// lambda_dt from the five dot products (fixed summation order), and the winning limit as
// step_begin_kernel chooses it.
// One block of kSumThreads: a fixed summation order (deterministic), many loads in flight.
constexpr int kSumThreads = 1024;
__global__ void __launch_bounds__(kSumThreads) adj_dt_sum_kernel(r3dk::Physics ph, const double* dots, int nblocks,
                                                                  double c0, double c1, double c2, double c3,
                                                                  double c4, AdjScalars* aux) {
    __shared__ double red[kSumThreads];
    const double coef[kDots] = {c0, c1, c2, c3, c4};
    double s = 0.0;
    for (int d = 0; d < kDots; ++d) {
        double p = 0.0;
        for (int b = threadIdx.x; b < nblocks; b += blockDim.x) p += dots[(size_t)d * nblocks + b];
        s += coef[d] * p;
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = kSumThreads / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        aux->lam_dt = red[0];
        const double w0 = r3dk::order_value(aux->wkey[0]), w1 = r3dk::order_value(aux->wkey[1]);
        const double w2 = r3dk::order_value(aux->wkey[2]), w3 = r3dk::order_value(aux->wkey[3]);
        int t = 0;
        double m = w0;
        if (w1 < m) { t = 1; m = w1; }
        if (w2 < m) { t = 2; m = w2; }
        if (ph.lmag && w3 < m) { t = 3; m = w3; }
        aux->term = t;
        aux->mstar = m;
        aux->argmin = ~0ull;
    }
}

__global__ void __launch_bounds__(BX* BY) adj_argmin_kernel(r3dk::Geometry g, r3dk::Physics ph, r3dk::Lines L,
                                                             AdjArgs A, AdjScalars* aux) {
    const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
    const int k = 1 + blockIdx.z;
    if (i > g.npx || j > g.npy) return;
    const int term = aux->term;
    if (term == 3) return;  // the constant magnetic-diffusion limit has no derivative
    const int n = k * (int)g.plane + j * (int)g.pitch + i;
    double b2 = 0.0;
    if (ph.lmag) {
        const double bx = A.x[5][n], by = A.x[6][n], bz = A.x[7][n];
        b2 = bx * bx + by * by + bz * bz;
    }
    const double dxy = (L.ddy[j] < L.ddx[i]) ? L.ddy[j] : L.ddx[i];
    const double dd = (L.ddz[k] < dxy) ? L.ddz[k] : dxy;  // the dt_full_kernel expression
    double w1, w2, w3, w4, um;
    r3dk::dt_terms(ph, A.x[0][n], A.x[1][n], A.x[2][n], A.x[3][n], A.x[4][n], b2, dd, L.rkapa[k], w1, w2, w3,
                   w4, um);
    const double wq = term == 0 ? w1 : (term == 1 ? w2 : w3);
    if (wq == aux->mstar) atomicMin(&aux->argmin, (unsigned long long)n);
}

__global__ void adj_dt_apply_kernel(r3dk::Geometry g, r3dk::Physics ph, r3dk::Lines L, AdjArgs A,
                                    AdjScalars* aux) {
    const unsigned long long an = aux->argmin;
    if (aux->term == 3 || an == ~0ull) return;
    const int n = (int)an;
    const int k = n / (int)g.plane, j = (n % (int)g.plane) / (int)g.pitch, i = n % (int)g.pitch;
    const double dxy = (L.ddy[j] < L.ddx[i]) ? L.ddy[j] : L.ddx[i];
    const double dd = (L.ddz[k] < dxy) ? L.ddz[k] : dxy;
    double xv[r3dk::kMaxFields], gv[r3dk::kMaxFields];
    for (int f = 0; f < A.nf; ++f) xv[f] = A.x[f][n];
    r3dk::adj_dt_cell(ph, aux->term, dd, L.rkapa[k], xv, A.nf, aux->lam_dt * ph.sff, gv);
    for (int f = 0; f < A.nf; ++f) A.lam[f][n] += gv[f];
}

// Count interior values that differ (bitwise) between a recomputed and a recorded state.
__global__ void __launch_bounds__(BX* BY) adj_compare_kernel(r3dk::Geometry g, const double* a, const double* b,
                                                              int64_t field_elems, int nf, AdjScalars* aux) {
    const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
    const int k = 1 + blockIdx.z;
    if (i > g.npx || j > g.npy) return;
    const int64_t n = (int64_t)k * g.plane + (int64_t)j * g.pitch + i;
    unsigned long long bad = 0;
    for (int f = 0; f < nf; ++f)
        bad += (__double_as_longlong(a[f * field_elems + n]) != __double_as_longlong(b[f * field_elems + n]));
    if (bad) atomicAdd(&aux->mismatch, bad);
}

}  // namespace

namespace r3dg {

// A state: nf fields stored back to back, field f at base + f*field_elems (padded layout).
struct StateBuf {
    double* base = nullptr;
    r3dk::StageMaps maps{};
};

struct Adjoint {
    int nf = 5;
    int64_t field_elems = 0;
    StateBuf S[4];                  // X_0 .. X_3 of the step being reversed
    double* Zb = nullptr;           // accumulator Z (nf fields)
    double* F[3] = {};              // F_0 .. F_2 (nf fields each)
    double* lam = nullptr;          // lambda_X (nf fields)
    double* lamF[2] = {};           // lambda_F, two buffers
    double* Lam = nullptr;          // pass-1 arrays
    int nlam = 0;
    double* dots = nullptr;
    int nblocks = 0;
    r3dk::Scalars* asc = nullptr;   // scalars of the recompute
    AdjScalars* aux = nullptr;
    AdjScalars* haux = nullptr;     // pinned mirror
    std::vector<double*> ckpt;      // recorded checkpoints
    std::vector<double*> seg;       // states of the segment being reversed
    int nsteps = 0, every = 0;
    bool recorded = false;
    int64_t bytes = 0;
};

namespace impl {

double* dalloc(Adjoint* A, size_t n) {
    double* p = nullptr;
    cuda_ok(cudaMalloc(&p, n * sizeof(double)), "cudaMalloc(adjoint)");
    A->bytes += (int64_t)(n * sizeof(double));
    return p;
}

double* state_field(double* base, const Adjoint* A, int f) { return base + (size_t)f * A->field_elems; }

dim3 cell_grid(const r3d_gpu* g) {
    return dim3((g->geo.npx + BX - 1) / BX, (g->geo.npy + BY - 1) / BY, (unsigned)g->geo.npz);
}

Adjoint* workspace(r3d_gpu* g) {
    if (g->adj) return g->adj;
    if (g->fp32) throw Error(R3D_EINVAL, "the adjoint is available for precision fp64 only");
    if (g->p.id != 0) throw Error(R3D_EINVAL, "the adjoint does not include the density diffusion (ID)");
    if (g->p.itcon == 2 || g->p.itcon == 3)
        throw Error(R3D_EINVAL, "the adjoint covers itcon 0, 1 and 4 (not the embedded heat loss or a free top T)");
    if (g->nloc != g->p.npz || g->halo) throw Error(R3D_EINVAL, "the adjoint needs the whole domain on one handle");
    if (g->p.tp != 0.0 && g->p.tc != 0.0 && (g->p.itcon == 0 || g->p.itcon == 1))
        throw Error(R3D_EINVAL, "the adjoint needs a time-independent top boundary (tc == 0)");
    if (g->geo.npz > 65535) throw Error(R3D_EINVAL, "the adjoint supports npz <= 65535");
    auto A = new Adjoint();
    try {
        A->nf = g->nfields;
        A->field_elems = g->geo.plane * (g->geo.npz + 2);
        const size_t st = (size_t)A->nf * A->field_elems;
        unsigned bx = 0, by = 0;
        r3dk::stage_fp64_box(g->geo.tile_rows, &bx, &by);
        for (int s = 0; s < 4; ++s) {
            A->S[s].base = dalloc(A, st);
            for (int f = 0; f < A->nf; ++f)
                A->S[s].maps.m[f] = field_map(state_field(A->S[s].base, A, f), g->d.nx, g->d.ny, g->d.nz,
                                              g->geo.pitch, g->geo.plane, bx, by,
                                              CU_TENSOR_MAP_DATA_TYPE_FLOAT64, sizeof(double));
        }
        A->Zb = dalloc(A, st);
        for (int s = 0; s < 3; ++s) A->F[s] = dalloc(A, st);
        A->lam = dalloc(A, st);
        for (int s = 0; s < 2; ++s) A->lamF[s] = dalloc(A, st);
        A->nlam = A->nf == 8 ? r3dk::kLamMax : r3dk::kLamHydro;
        A->Lam = dalloc(A, (size_t)A->nlam * A->field_elems);
        const dim3 gr = cell_grid(g);
        A->nblocks = (int)(gr.x * gr.y * gr.z);
        A->dots = dalloc(A, (size_t)kDots * A->nblocks);
        cuda_ok(cudaMalloc(&A->asc, sizeof(r3dk::Scalars)), "cudaMalloc(adjoint scalars)");
        cuda_ok(cudaMemsetAsync(A->asc, 0, sizeof(r3dk::Scalars), g->stream), "cudaMemset");
        cuda_ok(cudaMalloc(&A->aux, sizeof(AdjScalars)), "cudaMalloc(adjoint scalars)");
        cuda_ok(cudaMemsetAsync(A->aux, 0, sizeof(AdjScalars), g->stream), "cudaMemset");
        cuda_ok(cudaMallocHost(&A->haux, sizeof(AdjScalars)), "cudaMallocHost");
        // F, Lambda and the lambda buffers are read at ghost-free interior cells only, but keep
        // every buffer defined
        for (double* p : {A->Zb, A->F[0], A->F[1], A->F[2], A->lam, A->lamF[0], A->lamF[1]})
            cuda_ok(cudaMemsetAsync(p, 0, st * sizeof(double), g->stream), "cudaMemset");
        cuda_ok(cudaMemsetAsync(A->Lam, 0, (size_t)A->nlam * A->field_elems * sizeof(double), g->stream),
                "cudaMemset");
    } catch (...) {
        g->adj = A;
        adjoint_free(g);
        throw;
    }
    g->adj = A;
    return A;
}

void free_states(std::vector<double*>& v) {
    for (double* p : v) cudaFree(p);
    v.clear();
}

// Copy the simulation's current state (separate field arrays) into a contiguous state buffer.
void save_current(r3d_gpu* g, Adjoint* A, double* dst) {
    const size_t nb = (size_t)A->field_elems * sizeof(double);
    for (int f = 0; f < A->nf; ++f)
        cuda_ok(cudaMemcpyAsync(state_field(dst, A, f), g->X[g->cur][f], nb, cudaMemcpyDeviceToDevice, g->stream),
                "checkpoint copy");
}

void copy_state(r3d_gpu* g, Adjoint* A, double* dst, const double* src) {
    if (dst == src) return;
    cuda_ok(cudaMemcpyAsync(dst, src, (size_t)A->nf * A->field_elems * sizeof(double), cudaMemcpyDeviceToDevice,
                            g->stream),
            "state copy");
}

r3dk::FieldSet stage_fields(const Adjoint* A, int s) {
    r3dk::FieldSet fs{};
    for (int f = 0; f < A->nf; ++f) {
        fs.xin[f] = state_field(A->S[s].base, A, f);
        fs.xout[f] = state_field(A->S[s + 1].base, A, f);
        fs.z[f] = state_field(A->Zb, A, f);
        fs.f[f] = state_field(A->F[s], A, f);
    }
    return fs;
}

// One forward step from S[0] (a copy of src) with every intermediate kept: S[1..3], F[0..2],
// and the limits/dt of the step in asc/aux.
void recompute_step(r3d_gpu* g, Adjoint* A, const double* src) {
    copy_state(g, A, A->S[0].base, src);
    cuda_ok(r3dk::launch_reset_reduction(A->asc, g->stream), "adjoint reset");
    r3dk::FieldSet f0 = stage_fields(A, 0);
    cuda_ok(r3dk::launch_dt_full(g->geo, g->ph, g->lines, f0, A->asc, g->stream), "adjoint dt_full");
    adj_save_limits_kernel<<<1, 1, 0, g->stream>>>(A->asc, A->aux);
    cuda_ok(cudaGetLastError(), "adjoint save limits");
    cuda_ok(r3dk::launch_step_begin(g->ph, A->asc, g->stream), "adjoint step_begin");
    for (int s = 0; s < 3; ++s) {
        r3dk::FieldSet fs = stage_fields(A, s);
        cuda_ok(r3dk::launch_stage_fp64(s, A->S[s].maps, g->geo, g->ph, g->lines, fs, A->asc, g->kchunk, g->stream,
                                        true),
                "adjoint recompute stage");
        cuda_ok(r3dk::launch_bcon(g->geo, g->ph, g->lines, g->bnd, fs, A->asc, 0, g->stream), "adjoint bcon");
    }
}

AdjArgs base_args(const r3d_gpu* g, const Adjoint* A) {
    AdjArgs a{};
    a.g = g->geo;
    a.ph = g->ph;
    a.L = g->lines;
    a.nf = A->nf;
    a.sc = A->asc;
    for (int q = 0; q < A->nlam; ++q) a.Lam[q] = A->Lam + (size_t)q * A->field_elems;
    for (int f = 0; f < A->nf; ++f) a.lam[f] = state_field(A->lam, A, f);
    return a;
}

// Reverse the step whose intermediates recompute_step left in the workspace: lam holds the
// adjoint of X_3 on entry and of X_0 on exit.
void reverse_step(r3d_gpu* g, Adjoint* A) {
    const dim3 blk(BX, BY, 1), cg = cell_grid(g);
    const dim3 cols((g->geo.npx + BX - 1) / BX, (g->geo.npy + BY - 1) / BY, 1);
    const double gam[3] = {g->ph.gam[0], g->ph.gam[1], g->ph.gam[2]};
    const double zeta[3] = {g->ph.zeta[0], g->ph.zeta[1], g->ph.zeta[2]};
    int cur = 0;
    for (int s = 2; s >= 0; --s) {
        AdjArgs a = base_args(g, A);
        for (int f = 0; f < A->nf; ++f) a.x[f] = state_field(A->S[s + 1].base, A, f);
        adj_bcon_kernel<<<cols, blk, 0, g->stream>>>(g->geo, g->ph, g->bnd, a);
        cuda_ok(cudaGetLastError(), "adj_bcon");
        double* lf[8] = {};
        for (int f = 0; f < A->nf; ++f) {
            lf[f] = state_field(A->lamF[cur], A, f);
            a.fprev[f] = state_field(A->F[s], A, f);
        }
        adj_seed_kernel<<<cg, blk, 0, g->stream>>>(a, lf[0], lf[1], lf[2], lf[3], lf[4], lf[5], lf[6], lf[7],
                                                   gam[s], s == 2 ? 1 : 0, A->dots + (size_t)(2 - s) * A->nblocks);
        cuda_ok(cudaGetLastError(), "adj_seed");
        AdjArgs p = base_args(g, A);
        for (int f = 0; f < A->nf; ++f) {
            p.x[f] = state_field(A->S[s].base, A, f);
            p.a[f] = lf[f];
            if (s > 0) {
                p.fnext[f] = state_field(A->lamF[1 - cur], A, f);
                p.fprev[f] = state_field(A->F[s - 1], A, f);
            }
        }
        p.zeta = zeta[s];
        adj_pass1_kernel<<<cg, blk, 0, g->stream>>>(p);
        cuda_ok(cudaGetLastError(), "adj_pass1");
        adj_pass2_kernel<<<cg, blk, 0, g->stream>>>(p, s > 0 ? A->dots + (size_t)(3 + (2 - s)) * A->nblocks : nullptr);
        cuda_ok(cudaGetLastError(), "adj_pass2");
        cur = 1 - cur;
    }
    adj_dt_sum_kernel<<<1, kSumThreads, 0, g->stream>>>(g->ph, A->dots, A->nblocks, gam[2], gam[1], gam[0], zeta[2], zeta[1],
                                               A->aux);
    cuda_ok(cudaGetLastError(), "adj_dt_sum");
    AdjArgs d = base_args(g, A);
    for (int f = 0; f < A->nf; ++f) d.x[f] = state_field(A->S[0].base, A, f);
    adj_argmin_kernel<<<cg, blk, 0, g->stream>>>(g->geo, g->ph, g->lines, d, A->aux);
    cuda_ok(cudaGetLastError(), "adj_argmin");
    adj_dt_apply_kernel<<<1, 1, 0, g->stream>>>(g->geo, g->ph, g->lines, d, A->aux);
    cuda_ok(cudaGetLastError(), "adj_dt_apply");
}

void compare_states(r3d_gpu* g, Adjoint* A, const double* a, const double* b) {
    const dim3 blk(BX, BY, 1), cg = cell_grid(g);
    adj_compare_kernel<<<cg, blk, 0, g->stream>>>(g->geo, a, b, A->field_elems, A->nf, A->aux);
    cuda_ok(cudaGetLastError(), "adj_compare");
}

// Host cotangent (NX*NY*NZ per field, ghosts included) -> lam: x/y ghost entries are added to
// the interior cells they image, z ghost planes are constants and dropped.
void upload_seed(r3d_gpu* g, Adjoint* A, const double* const* seed) {
    const int64_t NX = g->d.nx, NY = g->d.ny, NZ = g->d.nz;
    const int npx = g->p.npx, npy = g->p.npy;
    std::vector<double> plane((size_t)g->geo.plane * NZ);
    auto wrap = [](int64_t q, int64_t np) { return q == 0 ? np : (q == np + 1 ? 1 : q); };
    for (int f = 0; f < A->nf; ++f) {
        if (!seed[f]) throw std::invalid_argument("null seed field");
        std::fill(plane.begin(), plane.end(), 0.0);
        for (int64_t k = 1; k <= NZ - 2; ++k)
            for (int64_t j = 0; j < NY; ++j)
                for (int64_t i = 0; i < NX; ++i) {
                    const double v = seed[f][(k * NY + j) * NX + i];
                    if (v == 0.0) continue;
                    const int64_t ii = wrap(i, npx), jj = wrap(j, npy);
                    plane[(size_t)(k * g->geo.plane + jj * g->geo.pitch + ii)] += v;
                }
        cuda_ok(cudaMemcpyAsync(state_field(A->lam, A, f), plane.data(), plane.size() * sizeof(double),
                                cudaMemcpyHostToDevice, g->stream),
                "seed upload");
        cuda_ok(cudaStreamSynchronize(g->stream), "seed upload");
    }
}

void download_grad(r3d_gpu* g, Adjoint* A, double* const* grad) {
    const int64_t NX = g->d.nx, NY = g->d.ny, NZ = g->d.nz;
    std::vector<double> plane((size_t)g->geo.plane * NZ);
    for (int f = 0; f < A->nf; ++f) {
        if (!grad[f]) throw std::invalid_argument("null gradient field");
        cuda_ok(cudaMemcpyAsync(plane.data(), state_field(A->lam, A, f), plane.size() * sizeof(double),
                                cudaMemcpyDeviceToHost, g->stream),
                "gradient download");
        cuda_ok(cudaStreamSynchronize(g->stream), "gradient download");
        for (int64_t k = 0; k < NZ; ++k)
            for (int64_t j = 0; j < NY; ++j)
                for (int64_t i = 0; i < NX; ++i) {
                    const bool inner = k >= 1 && k <= NZ - 2 && j >= 1 && j <= NY - 2 && i >= 1 && i <= NX - 2;
                    grad[f][(k * NY + j) * NX + i] =
                        inner ? plane[(size_t)(k * g->geo.plane + j * g->geo.pitch + i)] : 0.0;
                }
    }
}

void check_aux(r3d_gpu* g, Adjoint* A) {
    cuda_ok(cudaMemcpyAsync(A->haux, A->aux, sizeof(AdjScalars), cudaMemcpyDeviceToHost, g->stream), "adjoint scalars");
    r3dk::Scalars sc{};
    cuda_ok(cudaMemcpyAsync(&sc, A->asc, sizeof(sc), cudaMemcpyDeviceToHost, g->stream), "adjoint scalars");
    cuda_ok(cudaStreamSynchronize(g->stream), "adjoint");
    if (sc.err != r3dk::kErrNone)
        throw Error(R3D_ECUDA, "a recompute stage kernel abandoned a bounded TMA wait; the gradient is invalid");
    if (A->haux->mismatch)
        throw Error(R3D_ENUMERIC, "adjoint recompute diverged from the recorded trajectory (" +
                                      std::to_string(A->haux->mismatch) + " values)");
}

}  // namespace impl

void adjoint_free(r3d_gpu* g) {
    Adjoint* A = g->adj;
    if (!A) return;
    for (auto& s : A->S) cudaFree(s.base);
    cudaFree(A->Zb);
    for (double* p : A->F) cudaFree(p);
    cudaFree(A->lam);
    for (double* p : A->lamF) cudaFree(p);
    cudaFree(A->Lam);
    cudaFree(A->dots);
    cudaFree(A->asc);
    cudaFree(A->aux);
    if (A->haux) cudaFreeHost(A->haux);
    impl::free_states(A->ckpt);
    impl::free_states(A->seg);
    delete A;
    g->adj = nullptr;
}

}  // namespace r3dg

using namespace r3dg;
using namespace r3dg::impl;

extern "C" {

int r3d_gpu_adjoint_record(r3d_gpu* g, int nsteps, int checkpoint_every, r3d_scalars* sc) {
    return guarded([&] {
        if (!g) throw std::invalid_argument("null handle");
        if (!g->uploaded) throw Error(R3D_ESTATE, "record before upload");
        if (nsteps < 1 || checkpoint_every < 1) throw std::invalid_argument("nsteps and checkpoint_every must be >= 1");
        DeviceGuard dg(g->device);
        Range r("r3d.adjoint_record");
        Adjoint* A = workspace(g);
        A->recorded = false;
        free_states(A->ckpt);
        // checkpoints at steps 0, K, 2K, .. and the final state (compared against in backward)
        const int nck = (nsteps + checkpoint_every - 1) / checkpoint_every + 1;
        const size_t st = (size_t)A->nf * A->field_elems;
        for (int c = 0; c < nck; ++c) {
            double* p = nullptr;
            cuda_ok(cudaMalloc(&p, st * sizeof(double)), "cudaMalloc(checkpoint)");
            A->ckpt.push_back(p);
        }
        Timer tm{g, false, nullptr};
        int launches = 0, stage_launches = 0;
        for (int n = 0; n < nsteps; ++n) {
            if (n % checkpoint_every == 0) save_current(g, A, A->ckpt[n / checkpoint_every]);
            enqueue_step(g, 3, tm, launches, stage_launches);
        }
        save_current(g, A, A->ckpt.back());
        pull_scalars(g, sc);
        A->nsteps = nsteps;
        A->every = checkpoint_every;
        A->recorded = true;
    });
}

int r3d_gpu_adjoint_backward(r3d_gpu* g, const double* const* seed, double* const* grad) {
    return guarded([&] {
        if (!g || !seed || !grad) throw std::invalid_argument("null argument");
        if (!g->adj || !g->adj->recorded) throw Error(R3D_ESTATE, "no recorded trajectory (call r3d_gpu_adjoint_record)");
        DeviceGuard dg(g->device);
        Range r("r3d.adjoint_backward");
        Adjoint* A = g->adj;
        const size_t st = (size_t)A->nf * A->field_elems;
        // the recompute buffers start as copies of X_0: their z ghost planes are constants
        for (int s = 1; s < 4; ++s) copy_state(g, A, A->S[s].base, A->ckpt[0]);
        cuda_ok(cudaMemsetAsync(&A->aux->mismatch, 0, sizeof(unsigned long long), g->stream), "cudaMemset");
        upload_seed(g, A, seed);
        const int K = A->every, N = A->nsteps;
        while ((int)A->seg.size() < K) {
            double* p = nullptr;
            cuda_ok(cudaMalloc(&p, st * sizeof(double)), "cudaMalloc(segment)");
            A->seg.push_back(p);
        }
        const double* final_state = A->ckpt.back();  // the recorded final state
        {
            const int nseg = (N + K - 1) / K;
            for (int sg = nseg - 1; sg >= 0; --sg) {
                const int s0 = sg * K, len = std::min(K, N - s0);
                copy_state(g, A, A->seg[0], A->ckpt[sg]);
                for (int s = 1; s < len; ++s) {
                    recompute_step(g, A, A->seg[s - 1]);
                    copy_state(g, A, A->seg[s], A->S[3].base);
                }
                for (int s = len - 1; s >= 0; --s) {
                    recompute_step(g, A, A->seg[s]);
                    const double* next = s + 1 < len ? A->seg[s + 1] : (sg + 1 < nseg ? A->ckpt[sg + 1] : final_state);
                    compare_states(g, A, A->S[3].base, next);
                    reverse_step(g, A);
                }
                check_aux(g, A);
            }
            download_grad(g, A, grad);
        }
    });
}

int r3d_gpu_adjoint_step(r3d_gpu* g, const double* const* seed, double* const* grad) {
    return guarded([&] {
        if (!g || !seed || !grad) throw std::invalid_argument("null argument");
        if (!g->uploaded) throw Error(R3D_ESTATE, "adjoint before upload");
        DeviceGuard dg(g->device);
        Adjoint* A = workspace(g);
        save_current(g, A, A->S[0].base);
        for (int s = 1; s < 4; ++s) copy_state(g, A, A->S[s].base, A->S[0].base);
        upload_seed(g, A, seed);
        recompute_step(g, A, A->S[0].base);
        reverse_step(g, A);
        check_aux(g, A);
        download_grad(g, A, grad);
    });
}

int r3d_gpu_adjoint_memory(const r3d_gpu* g, int64_t* bytes) {
    return guarded([&] {
        if (!g || !bytes) throw std::invalid_argument("null argument");
        const Adjoint* A = g->adj;
        int64_t b = 0;
        if (A) {
            const int64_t st = (int64_t)A->nf * A->field_elems * (int64_t)sizeof(double);
            b = A->bytes + st * (int64_t)(A->ckpt.size() + A->seg.size());
        }
        *bytes = b;
    });
}

}  // extern "C"
