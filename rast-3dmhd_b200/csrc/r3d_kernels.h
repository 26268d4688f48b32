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

size_t stage_fp64_smem();
// TMA box (x, y) of one field plane that the FP64 stage kernel was compiled for.
void stage_fp64_box(unsigned* bx, unsigned* by);
cudaError_t launch_stage_fp64(int stage, const StageMaps& maps, const Geometry& g,
                              const Physics& ph, const Lines& L, const FieldSet& fs, Scalars* sc,
                              int kchunk, cudaStream_t st);
cudaError_t launch_bcon(const Geometry& g, const Physics& ph, const Lines& L, const Boundary& b,
                        const FieldSet& fs, Scalars* sc, int with_dt, cudaStream_t st);
cudaError_t launch_dt_full(const Geometry& g, const Physics& ph, const Lines& L,
                           const FieldSet& fs, Scalars* sc, cudaStream_t st);
cudaError_t launch_step_begin(const Physics& ph, Scalars* sc, cudaStream_t st);
cudaError_t launch_step_end(Scalars* sc, cudaStream_t st);
cudaError_t launch_reset_reduction(Scalars* sc, cudaStream_t st);
cudaError_t launch_totals(const Geometry& g, const Physics& ph, const FieldSet& fs, Scalars* sc,
                          cudaStream_t st);

}  // namespace r3dk
