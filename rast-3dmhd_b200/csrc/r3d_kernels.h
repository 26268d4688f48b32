// r3d_kernels.h - launchers of the step kernels (host side of csrc/*.cu).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "r3d_device.cuh"

namespace r3dk {

// Field pointers of one stage: the state read (xin), the state written (xout) and the RK
// accumulator read/written in place (z); order ru rv rw ro tt bx by bz.
struct FieldSet {
    const double* xin[kMaxFields];
    double* xout[kMaxFields];
    double* z[kMaxFields];
    double* f[kMaxFields];  // right-hand sides F, stored only by the adjoint's recompute launches
};

// FP32-bulk field pointers: thermodynamic deviations and momenta stored as float.
struct FieldSet32 {
    const float* xin[5];
    float* xout[5];
    float* z[5];
};

// TMA descriptors of the state fields read by a stage (ru rv rw ro tt, + bx by bz with MHD):
// a 3D map over (x, y, z) = (npx+2, npy+2, npz+2) doubles with the padded row pitch, one
// (34, TY+2, 1) box per plane.
struct StageMaps {
    CUtensorMap m[kMaxFields];
};

// Static background of the FP32-bulk form: R(k), T0(k) of the polytrope over the global z
// index (FP64 and FP32 copies) and the per-plane background parts of the z terms, in FP64:
// hres = g*R - (R*T0)_z (hydrostatic residual), dt0 = T0(k+1) - T0(k-1),
// lt0 = dt0*tmpz1 + (T0(k+1) - 2*T0(k) + T0(k-1))*tmpz2.
struct Background {
    const double *r, *t, *hres, *dt0, *lt0;
    const float *rf, *tf;
    const float4* kf;  // per plane, 3 x float4: {tmpz, tmpz1, tmpz2, hz*dzzdz}, {hres, dt0, lt0, rkapa},
                       // {dkapa, R, T0, 0}
};

void stage_fp32_box(unsigned* bx, unsigned* by);
// CTAs of the FP32-bulk stage kernel resident per SM (the chunk planner's slots).
int stage_fp32_ctas_per_sm();
cudaError_t launch_stage_fp32(int stage, const StageMaps& maps, const Geometry& g, const Physics& ph,
                              const Lines& L, const Background& bg, const FieldSet32& fs, Scalars* sc,
                              int kchunk, cudaStream_t st);
cudaError_t launch_bcon_fp32(const Geometry& g, const Physics& ph, const Lines& L, const Boundary& b,
                             const Background& bg, const FieldSet32& fs, Scalars* sc, int with_dt,
                             cudaStream_t st);
cudaError_t launch_dt_full_fp32(const Geometry& g, const Physics& ph, const Lines& L,
                                const Background& bg, const FieldSet32& fs, Scalars* sc, cudaStream_t st,
                                int only_refold = 0);
cudaError_t launch_totals_fp32(const Geometry& g, const Physics& ph, const Background& bg,
                               const FieldSet32& fs, Scalars* sc, cudaStream_t st);

size_t stage_fp64_smem();
// Rows of the FP64 stage kernel's column tiles for a grid (8 hydro; MHD 6, or 8 on grids too
// small for two CTAs per SM), and the TMA box (x, y) of one field plane for tiles of that height.
int stage_fp64_rows(int mhd, int npx, int npy, int nloc, int num_sms);
// resident CTAs per SM of the FP64 stage kernels (hydro: all three stages; MHD: by tile rows)
int stage_fp64_ctas_per_sm(int mhd, int rows);
// Horizontal means of rho per local plane (density diffusion): rom[k], and wwz[k] = 1/rom[k]
// when id_mode == 1; the domain's ghost planes take the means of their mirror planes.
cudaError_t launch_plane_mean(const Geometry& g, const double* ro, double* rom, double* wwz, int id_mode,
                              cudaStream_t st);
void stage_fp64_box(int rows, unsigned* bx, unsigned* by);
cudaError_t launch_stage_fp64(int stage, const StageMaps& maps, const Geometry& g,
                              const Physics& ph, const Lines& L, const FieldSet& fs, Scalars* sc,
                              int kchunk, cudaStream_t st, bool emit_rhs = false);
cudaError_t launch_bcon(const Geometry& g, const Physics& ph, const Lines& L, const Boundary& b,
                        const FieldSet& fs, Scalars* sc, int with_dt, cudaStream_t st);
// only_refold: run only if step_end requested a re-evaluation (Scalars::refold)
cudaError_t launch_dt_full(const Geometry& g, const Physics& ph, const Lines& L,
                           const FieldSet& fs, Scalars* sc, cudaStream_t st, int only_refold = 0);
cudaError_t launch_step_begin(const Physics& ph, Scalars* sc, cudaStream_t st);
// check: verify the filtered limits of a full step (Scalars::thr_*), request a refold if needed
cudaError_t launch_step_end(Scalars* sc, cudaStream_t st, int check = 0);
cudaError_t launch_reset_reduction(Scalars* sc, cudaStream_t st);
// copy the limit keys to Scalars::wloc/uloc (a slab, before its keys are combined with others')
cudaError_t launch_save_local_limits(Scalars* sc, cudaStream_t st);
cudaError_t launch_totals(const Geometry& g, const Physics& ph, const FieldSet& fs, Scalars* sc,
                          cudaStream_t st);

}  // namespace r3dk
