// C entry points of one copy of the reference's own GPU driver (test infrastructure only).
//
// oracle/Makefile builds src/gpu.cpp and src/gpu_kernels.cu unmodified, with the flags of the
// reference's gpu backend (makefile:104-109, 185-190: -O2 -std=c++17 -fmad=false -x cu
// -rdc=true, static cudart; the architecture sm_100a in place of its sm_90 default), and links
// them with this file into _ref/libr3dgpu_r<N>.so: one physical copy per thread-rank.  The
// driver keeps its staging buffers in function-level statics (src/gpu.cpp:406-459, 553-554,
// 684-685, 790), which ranks sharing one process would otherwise share; the harness
// (ref_harness.cpp) opens copy N with RTLD_LOCAL for rank N, so each rank has its own.  The
// copies resolve MPI_* against the thread-rank MPI stand-in in libr3dref.so.
#include <cuda_runtime_api.h>

#include "gpu.hpp"

extern "C" {

// gpu_alloc + the GpuSim it fills (src/gpu.cpp:185-230)
void* r3dg_alloc(const r3d::Derived* d) {
    auto* g = new r3d::GpuSim;
    r3d::gpu_alloc(*g, *d);
    return g;
}

void r3dg_upload(void* g, const r3d::SimState* s) { r3d::gpu_upload(*static_cast<r3d::GpuSim*>(g), *s); }

void r3dg_download(r3d::SimState* s, void* g) { r3d::gpu_download(*s, *static_cast<r3d::GpuSim*>(g)); }

// step_gpu(nstages, ...) (src/gpu.cpp:736-1047) on MPI_COMM_WORLD; `sc` is the scalar mirror
// (dt, nit, timc, timt, timi, tb), as src/main.cpp:241-264 passes it
void r3dg_step(int nstages, const r3d::Params* p, const r3d::Derived* d, const r3d::Topology* t, void* g,
               r3d::SimState* sc) {
    r3d::step_gpu(nstages, MPI_COMM_WORLD, *p, *d, *t, *static_cast<r3d::GpuSim*>(g), *sc);
}

void r3dg_free(void* g) {
    r3d::gpu_free(*static_cast<r3d::GpuSim*>(g));
    delete static_cast<r3d::GpuSim*>(g);
}

int r3dg_sync(void) { return (int)cudaDeviceSynchronize(); }

}  // extern "C"
