// r3d_gpu_impl.hpp - the device-side simulation object behind the opaque r3d_gpu handle, and
// the helpers shared by the forward entry points (r3d_gpu.cu) and the adjoint (adjoint.cu).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <cstdint>
#include <string>
#include <utility>
#include <vector>

#include "r3d_device.cuh"
#include "r3d_error.hpp"
#include "r3d_gpu.h"
#include "r3d_host.hpp"
#include "r3d_kernels.h"

namespace r3dg {
struct Adjoint;  // reverse-mode workspace, created on first use (adjoint.cu)
struct Halo;     // inter-process slab exchange (halo.cu)
}

struct r3d_gpu {
    r3d_params p;
    r3db::Derived d;
    int device = 0;
    int num_sms = 148;  // multiprocessors of the device (read at create)
    cudaStream_t stream = nullptr;
    r3dk::Geometry geo{};
    r3dk::Physics ph{};
    r3dk::Lines lines{};
    r3dk::Boundary bnd{};
    int nfields = 5;
    double* X[2][r3dk::kMaxFields] = {};
    r3dk::StageMaps maps[2];  // TMA maps of X[0] and X[1] (ru rv rw ro tt)
    double* Z[r3dk::kMaxFields] = {};
    // FP32-bulk state (precision == R3D_PREC_FP32BULK): momenta and rho', T' deviations
    bool fp32 = false;
    float* X32[2][5] = {};
    float* Z32[5] = {};
    r3dk::Background bg{};
    void* bg_buf = nullptr;
    double* line_buf = nullptr;
    r3dk::Scalars* dsc = nullptr;
    r3dk::Scalars* hsc = nullptr;  // pinned mirror
    int cur = 0;
    int kchunk = 32;
    bool uploaded = false;
    bool work_ok = false;  // the last operation on the state was a full step (r3d_gpu_download_work)
    int64_t bytes = 0;
    double host_timc = 0.0, host_timi = 0.0;  // host clock for the plume relaxation (tc != 0)
    std::vector<cudaEvent_t> ev;             // timing events (r3d_gpu_run_timed)
    r3dg::Adjoint* adj = nullptr;            // reverse-mode workspace (adjoint entry points)
    // z slab held by this handle: global planes z0+1 .. z0+nloc (the whole domain: 0, npz)
    int z0 = 0, nloc = 0;
    bool own_stream = true;
    r3dg::Halo* halo = nullptr;              // ghost-plane exchange with other slabs (NCCL)
    double* fscr = nullptr;                  // r3d_gpu_fluxes scratch: X', Z', F (nfields each)
    // threshold filter of the third stage's limits (on a slab: thresholds and check from the
    // slab's own limits, Scalars::thr_local)
    bool dt_filter = true;
    double thr_margin = 1.0 / 64.0;
    // two whole steps captured as a CUDA graph, one per state-buffer parity at capture (r3d_gpu_run
    // replays it; six stages leave the parity unchanged)
    cudaGraphExec_t step_graph[2] = {nullptr, nullptr};
    int64_t steps_enqueued = 0;
};

namespace r3dg {

inline void cuda_ok(cudaError_t e, const char* what) {
    if (e != cudaSuccess)
        throw r3db::Error(e == cudaErrorMemoryAllocation ? R3D_ENOMEM : R3D_ECUDA,
                          std::string(what) + ": " + cudaGetErrorString(e));
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int now = -1;
        cudaGetDevice(&now);
        if (prev >= 0 && now != prev) cudaSetDevice(prev);
    }
};

// NVTX range over a host scope ("r3d.step", "r3d.stage", ...), for profiler timelines; free
// when no tool is attached.
struct Range {
    explicit Range(const char* name) { nvtxRangePushA(name); }
    ~Range() { nvtxRangePop(); }
    Range(const Range&) = delete;
    Range& operator=(const Range&) = delete;
};

// CUDA-event spans of a queued step sequence (inactive when on == false).
struct Timer {
    r3d_gpu* g;
    bool on;
    r3d_timing* tm;
    std::vector<std::pair<int, int>> spans;  // (event index, category)
    int next = 0;
    cudaEvent_t at(int idx) {
        while ((int)g->ev.size() <= idx) {
            cudaEvent_t e;
            cuda_ok(cudaEventCreate(&e), "cudaEventCreate");
            g->ev.push_back(e);
        }
        return g->ev[idx];
    }
    void begin() {
        if (on) cuda_ok(cudaEventRecord(at(next), g->stream), "cudaEventRecord");
    }
    void end(int cat) {
        if (!on) return;
        cuda_ok(cudaEventRecord(at(next + 1), g->stream), "cudaEventRecord");
        spans.push_back({next, cat});
        next += 2;
    }
};

// 3D TMA map over one padded field: dims (nx, ny, nz), one (box_x, box_y, 1) box per copy.
CUtensorMap field_map(void* base, int64_t nx, int64_t ny, int64_t nz, int64_t pitch, int64_t plane,
                      cuuint32_t box_x, cuuint32_t box_y, CUtensorMapDataType type, size_t esize);
r3dk::FieldSet fieldset(const r3d_gpu* g);
void launch_dt_full_any(r3d_gpu* g, int only_refold = 0);
void enqueue_step(r3d_gpu* g, int nstages, Timer& tm, int& launches, int& stage_launches);
void pull_scalars(r3d_gpu* g, r3d_scalars* sc);

// Slab handles (a z range of the domain) and the pieces of one step, for drivers that
// interleave several slabs with their ghost-plane exchanges (mesh.cu, halo.cu).
r3d_gpu* create_handle(const r3d_params& p, int z0, int nloc, cudaStream_t shared_stream);
void destroy_handle(r3d_gpu* g);
void enqueue_step_begin(r3d_gpu* g);
void enqueue_stage(r3d_gpu* g, int s);  // stage s + BCON; the new state becomes current
void enqueue_step_end(r3d_gpu* g, int nstages);
// Device pointer and element size of field q of the current state (FP64 or FP32-bulk).
void* state_field(r3d_gpu* g, int q, size_t* esize);
int state_fields(const r3d_gpu* g);

// halo.cu
void halo_free(r3d_gpu* g);
void halo_reduce_limits(r3d_gpu* g);  // before step_begin: global min/max of the dt keys
void halo_exchange(r3d_gpu* g);       // after a stage: ghost planes from the z neighbours

// adjoint.cu
void adjoint_free(r3d_gpu* g);

}  // namespace r3dg
