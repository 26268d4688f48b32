/* r3d_gpu.h - C ABI of the B200 Rast-3DMHD time step (librast3d_b200.so).
 *
 * The reference binds its GPU step through C++ entry points in include/gpu.hpp:18-49
 * (gpu_alloc / gpu_upload / step_gpu / gpu_download / gpu_free) and its configuration through
 * include/params.hpp:24-158 (Params, Derived, parse_args).  This header is the same surface as
 * plain C: plain structs, pointers and sizes, status codes instead of exit(), so that any host
 * language can bind it.  Each entry point names the reference interface it replaces.
 *
 * Domain: one GPU holds the whole global domain that the reference splits over npey x npez MPI
 * ranks.  Host arrays exchanged through this ABI use the reference layout on the global domain:
 * (npx+2) x (npy+2) x (npz+2) doubles, x fastest, idx = i + NX*(j + NY*k), interior
 * i in [1,npx], j in [1,npy], k in [1,npz]; ghost cells at the ends of every axis.
 *
 * Errors: every call returns R3D_OK (0) or a negative R3D_E* code; r3d_last_error() returns a
 * message for the calling thread's most recent failure.  Nothing here calls exit().
 */
#ifndef R3D_GPU_H
#define R3D_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    R3D_OK = 0,
    R3D_EINVAL = -1,      /* bad argument / unsupported configuration */
    R3D_ECUDA = -2,       /* CUDA runtime error */
    R3D_ENOMEM = -3,      /* device or host allocation failed */
    R3D_ESTATE = -4,      /* call out of order (e.g. step before upload) */
    R3D_ENUMERIC = -5     /* non-finite dt or dt underflow detected by the step */
};

enum { R3D_PREC_FP64 = 0, R3D_PREC_FP32BULK = 1 };

/* Run configuration: every field of the reference Params (include/params.hpp:24-120) with the
 * same meaning and defaults, plus three extensions (seed, precision, stages_per_graph). */
typedef struct r3d_params {
    int npx, npy, npz, npey, ix, iy, ilap, ipad, ngrid, id, ncol, nrow;
    int ixcon, iycon, izcon, itcon, ibcon;
    int lrot, lmag, lpot, lrem, lshr;
    int ncase, ncasep, ntotal, nstep0, nstart, ntube;
    double re, pr, theta, grav, r_y, ang, rm, beta, pzp, sigma, polys, tp, tc, xp, yp, zp;
    double xmax, ymax, zmax, ampt, ampb, bfh, bzp, qfh, gamma, hh, dh, dv, tstart, toff, rlax;
    double xx1, xx2, yy1, yy2, zz1, zz2, xa, xb, xc, xd, ya, yb, yc, yd, za, zb, zc, zd;
    double xcent, zcent, rmax, cmt, a_tube, lambda, vz0, sf;
    int backend; /* 0 = cpu, 1 = gpu (reference --backend) */
    int gpu_id;  /* reference --gpu */
    /* extensions */
    int seed;      /* --seed N: RAN2 seed idum = -N (reference hard-wires N = 62659) */
    int precision; /* --precision fp64|fp32bulk */
} r3d_params;

/* Scalars the reference carries in SimState (include/fields.hpp:137-143). */
typedef struct r3d_scalars {
    double dt, timc, timt, timi, umach, tb;
    int nit;
} r3d_scalars;

/* Host view of the state on the global domain (see layout above).  3D arrays hold
 * NX*NY*NZ doubles; x/y/z lines hold NX/NY/NZ doubles.  bx/by/bz may be NULL when lmag = 0.
 * Mirrors the reference SimState primaries + 1D metrics (include/fields.hpp:75-145). */
typedef struct r3d_host_state {
    double *ru, *rv, *rw, *ro, *tt, *bx, *by, *bz;
    double *exx, *dxxdx, *d2xxdx2, *ddx;
    double *wyy, *dyydy, *d2yydy2, *ddy;
    double *zee, *dzzdz, *d2zzdz2, *ddz, *rkapa, *dkapa;
} r3d_host_state;

/* Per-kernel timing of r3d_gpu_run_timed (CUDA events on the library's stream). */
typedef struct r3d_timing {
    double total_ms;        /* whole run, first launch to last */
    double stage_ms;        /* sum over the fused stage kernels */
    double bcon_ms;         /* sum over BCON + ghost + dt-edge kernels */
    double other_ms;        /* dt finalise / scalar kernels */
    int stage_launches;
    int total_launches;     /* kernels launched by the library in the run */
} r3d_timing;

typedef struct r3d_gpu r3d_gpu;

/* ---- configuration (replaces Params defaults, parse_args, derive: src/params.cpp:14-266) ---- */
int r3d_params_default(r3d_params* p);
/* Parses reference flags ("--npx 32", "--lmag=1", ...) plus --seed and --precision on top of
 * *p.  Unknown flags are an error (R3D_EINVAL), as in the reference.  argv excludes argv[0]. */
int r3d_params_parse(int argc, const char* const* argv, r3d_params* p);
/* Validates p for this implementation (stencil widths 2, periodic x/y, supported toggles). */
int r3d_params_check(const r3d_params* p);
/* Derived constants by name ("c13", "hx", "repr", ...); mirrors Derived (include/params.hpp:125-145). */
int r3d_derived_get(const r3d_params* p, const char* name, double* out);
/* Global grid sizes NX, NY, NZ. */
int r3d_dims(const r3d_params* p, int64_t* nx, int64_t* ny, int64_t* nz);

/* ---- host set-up: grid metrics + conductivity + static IC + ghost fill (src/main.cpp:134-154,
 *      src/grid.cpp:148-284, src/static_ic.cpp:24-161, src/ode.cpp:152-174) ---------------- */
int r3d_setup_host(const r3d_params* p, r3d_host_state* st, r3d_scalars* sc);
/* The same for the z slab of r3d_gpu_create_slab: fields hold global planes z0 .. z0+nz+1 and
 * the z metric lines nz+2 entries from global index z0 (x/y lines in full); identical to the
 * corresponding part of r3d_setup_host (the RAN2 stream is advanced past the planes above). */
int r3d_setup_host_slab(const r3d_params* p, int z0, int nz, r3d_host_state* st, r3d_scalars* sc);
/* Static polytrope T(k), R(k), k = 0..npz-1 (src/ode.cpp:152-174). */
int r3d_static_profile(const r3d_params* p, double* t, double* r);

/* ---- device state (replaces gpu_alloc / gpu_upload / gpu_download / gpu_free,
 *      include/gpu.hpp:35-38) ----------------------------------------------------------- */
int r3d_gpu_create(const r3d_params* p, r3d_gpu** out);
/* A handle over the z slab of global planes z0+1 .. z0+nz (4 <= nz; the reference's npez
 * decomposition, src/topology.cpp): its host arrays hold nz+2 planes, global planes z0 .. z0+nz+1,
 * the outer two being the z neighbours' planes (or the domain's ghost planes); the z metric
 * lines are the global ones from index z0 on.  BCON and the one-sided edge stencils apply only
 * where the slab touches the domain's top or bottom.  On its own a slab handle sees its ghost
 * planes as constants; r3d_gpu_halo_init connects the slabs of several processes. */
int r3d_gpu_create_slab(const r3d_params* p, int z0, int nz, r3d_gpu** out);
int r3d_gpu_upload(r3d_gpu* g, const r3d_host_state* st, const r3d_scalars* sc);
/* The initial state built on the device (replaces r3d_setup_host + r3d_gpu_upload; the set-up
 * of src/main.cpp:134-154, src/static_ic.cpp:24-161): metric lines, static columns and the
 * magnetic layer from the host (1D), the fields filled by kernels, and the seeded temperature
 * perturbation streamed plane by plane - RAN2 is one sequential chain, drawn on the host into a
 * small pinned ring while the device applies the planes before.  No host 3D arrays.  The state
 * (and *sc: zeros and tb) is bit-identical to r3d_setup_host followed by r3d_gpu_upload; works
 * for slab handles (the draws of the planes above the slab are skipped) and both precisions. */
int r3d_gpu_setup(r3d_gpu* g, r3d_scalars* sc);
int r3d_gpu_download(r3d_gpu* g, r3d_host_state* st, r3d_scalars* sc);
/* The RK accumulators (the reference's ZRU ZRV ZRW ZRO ZTT, + ZBX ZBY ZBZ with lmag: the
 * SimState fields gpu_download fills, include/fields.hpp:118,123) into z[0..nfields-1] (NULL
 * entries skipped), host arrays in the layout of r3d_gpu_download.  Interior cells; after a
 * full step they hold X + zeta_2 dt F of the second stage, as after the reference's step()
 * (src/step.cpp:240-246).  Ghost cells are not maintained (0 or stale). */
int r3d_gpu_download_accumulators(r3d_gpu* g, double* const* z);
int r3d_gpu_destroy(r3d_gpu* g);
/* ---- z slabs over several processes (replaces the MPI/NCCL halo exchange of
 *      src/communicate.cpp:70-182 and the dt MPI_Allreduce of src/step.cpp:224) ----
 * One process per GPU, rank r holding the r-th slab in z order.  Rank 0 calls
 * r3d_nccl_unique_id and distributes the 128 bytes; every rank then calls r3d_gpu_halo_init
 * (collective).  From then on every step combines the dt limits of all slabs (ncclAllReduce on
 * the device) and exchanges the ghost planes after every stage (ncclSend/ncclRecv), all on the
 * library stream; results equal the single-domain run bit for bit.  NCCL is loaded at run time
 * (libnccl.so.2); R3D_EINVAL when it is absent. */
int r3d_nccl_unique_id(unsigned char* out, size_t len);
int r3d_gpu_halo_init(r3d_gpu* g, const unsigned char* id, size_t len, int rank, int nranks);

/* ---- the same decomposition inside one process (several slabs on one device) ----
 * nslabs slabs of npz/nslabs (+1) planes on device gpu_id, exchanging ghost planes by device
 * copies; upload/step/run/download take the global host state like r3d_gpu_*.  Needs tc == 0
 * when tp != 0 (one shared host clock is not kept). */
typedef struct r3d_mesh r3d_mesh;
int r3d_mesh_create(const r3d_params* p, int nslabs, r3d_mesh** out);
int r3d_mesh_slab(const r3d_mesh* m, int r, int* z0, int* nz);
int r3d_mesh_upload(r3d_mesh* m, const r3d_host_state* st, const r3d_scalars* sc);
int r3d_mesh_step(r3d_mesh* m, int nstages, r3d_scalars* sc);
int r3d_mesh_run(r3d_mesh* m, int nsteps, r3d_scalars* sc);
int r3d_mesh_download(r3d_mesh* m, r3d_host_state* st, r3d_scalars* sc);
int r3d_mesh_destroy(r3d_mesh* m);
/* Test hook: r3d_gpu_debug_dt_filter on every slab of the mesh; *refolds (may be NULL) receives
 * the refolds of all slabs together. */
int r3d_mesh_debug_dt_filter(r3d_mesh* m, double margin, int* refolds);

/* FLUXES (src/fluxes.cpp:44-533; with lmag the LMAG branch of 3dmhdsub.f:2146-2650) of the
 * current device state, without changing it: out = nfields host arrays (NX*NY*NZ) receiving
 * FU FV FW FR FT (+ the B fluxes WW1 WW2 WW3), interior cells, ghosts 0.  On the domain's top
 * and bottom planes the momentum and energy right-hand sides, which BCON overwrites, are
 * returned as 0; the continuity and B fluxes there are the reference's one-sided forms.
 * FP64 only; refused (R3D_EINVAL) with the density diffusion (ID), which exists only inside a
 * stage, after its per-plane means. */
int r3d_gpu_fluxes(r3d_gpu* g, double* const* out);

/* The FLUXES work arrays of the reference's gstate dump (src/main.cpp:80-83) as they stand after
 * a full step: out = 8 host arrays (NX*NY*NZ; any may be NULL) receiving UU VV WW FU FV FW FR FT
 * of the third stage's input state.  UU = RU * (1/RO) etc. over the whole local array, ghosts
 * included (src/fluxes.cpp:131-165); FU..FT as r3d_gpu_fluxes forms them (interior cells; on the
 * domain's top and bottom planes the momentum and energy entries are 0, where the reference keeps
 * right-hand sides that BCON then overrides).  R3D_ESTATE unless the last operation on the state
 * was a full 3-stage step; FP64 only; FU..FT are refused with density diffusion (ID).  The state
 * is unchanged. */
int r3d_gpu_download_work(r3d_gpu* g, double* const* out);

/* Test hook for the failure path: from the next step on, every TMA transaction of the stage
 * kernels expects `bytes` more than its copies deliver, so each bounded wait runs out (200 ms),
 * the kernel records the error and returns, and the step reports R3D_ECUDA; the context stays
 * usable.  0 (the default, restored by r3d_gpu_upload) switches it off. */
int r3d_gpu_debug_tma_extra(r3d_gpu* g, unsigned int bytes);

/* The third stage's time-step limits are folded through a filter: cells whose float estimates
 * of the CFL limit and Mach term lie clearly beyond the previous step's limits widened by a
 * relative margin (default 1/64) skip the exact FP64 evaluation, and when the folded result
 * fails the check that makes this exact, the limits are evaluated again over the whole state
 * (a "refold").  The dt is bit-identical either way.  Test hook: margin (NaN: unchanged) sets
 * the margin - a negative one makes every full step refold - and *refolds (may be NULL)
 * receives the number of refolds since the upload.  A z-slab handle (r3d_gpu_create_slab, the
 * mesh) takes its thresholds from its own limits, saved before they are combined with the
 * other slabs', and checks its own fold, so each slab's limits - and their minimum over the
 * slabs - stay exact. */
int r3d_gpu_debug_dt_filter(r3d_gpu* g, double margin, int* refolds);

/* Launch plan of the stage kernels for a handle created with *p over nloc local z planes (0:
 * the whole npz, as r3d_gpu_create) on a device with num_sms multiprocessors: *kchunk receives
 * the z planes each CTA marches through, *tile_rows the rows of its 32-column tile.  With
 * num_sms > 0 this is host-only (no device needed); num_sms <= 0 reads the SM count of device
 * p->gpu_id, as a handle does at create.  R3D_KCHUNK=<planes> in the environment (a whole
 * number, clamped to [1, nloc]) overrides the depth, as it does for a handle.  The depth starts at 64
 * planes (npz >= 512), 32 (>= 256) or 16; MHD with 32x6 tiles takes 12; a launch that does not
 * fill the GPU once takes the depth (down to 4) minimising waves x planes per chunk; a hydro
 * launch of up to 64 waves takes a slightly shallower depth (at most one chunk more) when a
 * list-scheduling estimate of the launch, whose last chunk's CTAs run last, finds it 0.5%
 * shorter. */
int r3d_gpu_plan(const r3d_params* p, int nloc, int num_sms, int* kchunk, int* tile_rows);

/* Bytes of device memory held by g. */
int r3d_gpu_memory(const r3d_gpu* g, int64_t* bytes);
/* The CUDA stream (cudaStream_t) every kernel of g is launched on. */
void* r3d_gpu_stream(r3d_gpu* g);

/* ---- time step (replaces step_gpu(comm, p, d, t, g, scalars) and step_gpu(nstages, ...),
 *      include/gpu.hpp:43-49; semantics of step(), src/step.cpp:114-257) ------------------ */
/* One RK3 step (nstages = 3) or its first nstages substages; updates *sc like the reference
 * (dt, umach, nit, timc, timt).  Synchronises with the device to return the scalars. */
int r3d_gpu_step(r3d_gpu* g, int nstages, r3d_scalars* sc);
/* nsteps full steps queued back to back with no host synchronisation in between (unless the
 * plume relaxation tc != 0 needs the host clock); then synchronises and returns scalars. */
int r3d_gpu_run(r3d_gpu* g, int nsteps, r3d_scalars* sc);
/* As r3d_gpu_run without the final synchronisation (sc may be NULL; scalars stay on device). */
int r3d_gpu_enqueue(r3d_gpu* g, int nsteps);
/* As r3d_gpu_run, recording CUDA events around every kernel launch into *tm. */
int r3d_gpu_run_timed(r3d_gpu* g, int nsteps, r3d_scalars* sc, r3d_timing* tm);

/* ---- FP32-bulk extras ---- */
/* Volume sums of rho and of the total energy proxy over the interior, accumulated in FP64 on
 * the device (mass = sum rho, energy = sum (rho*T*cv + 0.5*(ru^2+rv^2+rw^2)/rho)). */
int r3d_gpu_totals(r3d_gpu* g, double* mass, double* energy);
/* Error norms of a's current state against ref's over the interior cells, computed on the
 * device (no counterpart in the reference; it measures the FP32-bulk form against FP64 on grids
 * whose host copies would not fit in host memory).  For each field q of ref (ru rv rw ro tt,
 * then bx by bz with lmag): out[4q..4q+3] = sum (a-ref)^2, sum ref^2, max |a-ref|, max |ref|.
 * Either handle may hold either precision (FP32-bulk rho and T compared as full values); both
 * must hold the same grid and slab on the same device.  Deterministic (fixed summation order). */
int r3d_gpu_compare(const r3d_gpu* a, const r3d_gpu* ref, double* out);

/* ---- discrete adjoint of the RK3 step (FP64; no counterpart in the reference) ----
 * Reverse-mode derivative of exactly the map r3d_gpu_run computes (FLUXES, the stage update,
 * BCON, the periodic ghost images and the dt minimum of src/step.cpp:114-257), with state
 * checkpoints on the device.  Cotangent arrays use the host layout of r3d_host_state fields:
 * one pointer per field in the order ru rv rw ro tt (+ bx by bz with lmag), each NX*NY*NZ
 * doubles.  Requires precision FP64 and a time-independent top boundary (tc == 0), else
 * R3D_EINVAL.  The derivative is taken w.r.t. the interior values of the starting state, whose
 * x/y ghost cells are the periodic images of the interior (as upload and every step leave
 * them); gradients are returned on interior cells, ghost entries 0.  dt = sff*min(limits)
 * contributes the derivative of the limit at the cell that sets it (lowest cell index on a
 * tie); at a cell at rest the momentum derivative of the CFL limit is taken as 0. */
/* Run nsteps (>= 1) forward from the current device state, as r3d_gpu_run does, keeping the
 * state every checkpoint_every steps (and the final state) for r3d_gpu_adjoint_backward.  The
 * simulation is left at the final state; later steps do not disturb the recording. */
int r3d_gpu_adjoint_record(r3d_gpu* g, int nsteps, int checkpoint_every, r3d_scalars* sc);
/* Given the cotangent of the recorded final state (seed), the cotangent of the recorded
 * starting state (grad).  Each segment is recomputed from its checkpoint; a recomputed state
 * that differs from the recorded one by a single bit gives R3D_ENUMERIC. */
int r3d_gpu_adjoint_backward(r3d_gpu* g, const double* const* seed, double* const* grad);
/* One-step vector-Jacobian product at the current device state (the state is not advanced). */
int r3d_gpu_adjoint_step(r3d_gpu* g, const double* const* seed, double* const* grad);
/* Device bytes held by the adjoint workspace and checkpoints (0 before first use). */
int r3d_gpu_adjoint_memory(const r3d_gpu* g, int64_t* bytes);

/* ---- allocation-free time-step limits (no counterpart in the reference) ----
 * For callers that cannot call cudaMalloc (for example a program that reserves the GPU's memory
 * in its own pool up front, or a time loop that must not pay the device synchronisation that
 * cudaMalloc/cudaFree may imply): computes {dt, umach} of a state the caller already holds in
 * device memory, as the next step would (src/step.cpp:122-229), using a fixed file-scope device
 * array for its partial results instead of allocated scratch.
 *   fields: 8 device pointers ru rv rw ro tt bx by bz (bx..bz only read when lmag), each the
 *           global (npx+2)(npy+2)(npz+2) array in the layout above;
 *   lines:  4 device pointers ddx[npx+2], ddy[npy+2], ddz[npz+2], rkapa[npz+2];
 *   out:    device pointer to 2 doubles, receives dt and umach;
 *   stream: cudaStream_t to launch on (NULL = legacy default stream); runs on device p->gpu_id.
 * Limit: ceil(npx/32)*ceil(npy/8) <= 65536 column tiles and ceil(npy/8) <= 65535, else
 * R3D_EINVAL.  Calls share the array, so calls that overlap on the GPU race.  Each call looks up
 * the array's address in the current context; the first call on a device also loads the module
 * there and should come before any stream capture.  Allocates no device memory. */
int r3d_dt_limits_noalloc(const r3d_params* p, const double* const* fields,
                          const double* const* lines, double* out, void* stream);

/* Message of the calling thread's last failed call ("" if none). */
const char* r3d_last_error(void);
/* Library version string. */
const char* r3d_version(void);

#ifdef __cplusplus
}
#endif
#endif
