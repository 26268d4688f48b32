// mesh.cu - the z-slab decomposition inside one process: several slab handles on one device,
// with the ghost-plane exchange done by device-to-device copies and the dt keys combined by a
// one-thread kernel.
//
// It runs exactly the sequence a multi-process run performs over NCCL (halo.cu) - per step:
// combine the limit keys of all slabs, step_begin on each, then for each stage the stage kernel
// and BCON on each slab followed by the exchange of every slab's first and last planes into
// its neighbours' ghost planes - so it checks the decomposition (slab-local BCON and one-sided
// stencils, ghost planes, the dt reduction) on a single GPU: every slab count must reproduce the
// single-domain state bit for bit.  It is also the form to use when one domain is to be split
// on one device (for example to mirror the reference's npez decomposition).
#include <cuda_runtime.h>

#include <vector>

#include "r3d_gpu_impl.hpp"

using namespace r3db;
using namespace r3dg;

struct r3d_mesh {
    r3d_params p;
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<r3d_gpu*> slabs;
    r3dk::Scalars** dsc = nullptr;  // device array of the slabs' scalar blocks
};

namespace {

__global__ void mesh_reduce_kernel(r3dk::Scalars** s, int n) {
    for (int r = 0; r < n; ++r) {  // each slab's own limits, for its dt filter thresholds
        for (int q = 0; q < 4; ++q) s[r]->wloc[q] = s[r]->wmin[q];
        s[r]->uloc = s[r]->umax;
    }
    unsigned long long w[4], u = s[0]->umax;
    for (int q = 0; q < 4; ++q) w[q] = s[0]->wmin[q];
    for (int r = 1; r < n; ++r) {
        for (int q = 0; q < 4; ++q) w[q] = s[r]->wmin[q] < w[q] ? s[r]->wmin[q] : w[q];
        u = s[r]->umax > u ? s[r]->umax : u;
    }
    for (int r = 0; r < n; ++r) {
        for (int q = 0; q < 4; ++q) s[r]->wmin[q] = w[q];
        s[r]->umax = u;
    }
}

void exchange(r3d_mesh* m) {
    Range r("r3d.mesh_exchange");
    for (size_t r = 0; r + 1 < m->slabs.size(); ++r) {
        r3d_gpu* a = m->slabs[r];
        r3d_gpu* b = m->slabs[r + 1];
        for (int q = 0; q < state_fields(a); ++q) {
            size_t es = 0;
            unsigned char* fa = static_cast<unsigned char*>(state_field(a, q, &es));
            unsigned char* fb = static_cast<unsigned char*>(state_field(b, q, &es));
            const size_t bytes = (size_t)a->geo.plane * es;
            cuda_ok(cudaMemcpyAsync(fb, fa + (size_t)a->nloc * bytes, bytes, cudaMemcpyDeviceToDevice, m->stream),
                    "ghost plane copy");
            cuda_ok(cudaMemcpyAsync(fa + (size_t)(a->nloc + 1) * bytes, fb + 1 * bytes, bytes,
                                    cudaMemcpyDeviceToDevice, m->stream),
                    "ghost plane copy");
        }
    }
}

void reduce(r3d_mesh* m) {
    mesh_reduce_kernel<<<1, 1, 0, m->stream>>>(m->dsc, (int)m->slabs.size());
    cuda_ok(cudaGetLastError(), "mesh reduce");
}

void mesh_step(r3d_mesh* m, int nstages) {
    reduce(m);
    for (r3d_gpu* g : m->slabs) enqueue_step_begin(g);
    for (int s = 0; s < nstages; ++s) {
        for (r3d_gpu* g : m->slabs) enqueue_stage(g, s);
        exchange(m);
    }
    for (r3d_gpu* g : m->slabs) enqueue_step_end(g, nstages);
}

// The slab's view of a host state on the global domain: planes z0 .. z0+nloc+1.
r3d_host_state slab_view(const r3d_host_state* st, const r3d_gpu* g) {
    const size_t off = (size_t)g->z0 * (size_t)(g->d.nx * g->d.ny);
    r3d_host_state v = *st;
    double** f[8] = {&v.ru, &v.rv, &v.rw, &v.ro, &v.tt, &v.bx, &v.by, &v.bz};
    for (double** p : f)
        if (*p) *p += off;
    double** z[6] = {&v.zee, &v.dzzdz, &v.d2zzdz2, &v.ddz, &v.rkapa, &v.dkapa};
    for (double** p : z)
        if (*p) *p += g->z0;
    return v;
}

void mesh_free(r3d_mesh* m) {
    for (r3d_gpu* g : m->slabs) destroy_handle(g);
    if (m->dsc) cudaFree(m->dsc);
    if (m->stream) cudaStreamDestroy(m->stream);
    delete m;
}

}  // namespace

extern "C" {

int r3d_mesh_create(const r3d_params* p, int nslabs, r3d_mesh** out) {
    return guarded([&] {
        if (!p || !out) throw std::invalid_argument("null argument");
        *out = nullptr;
        if (nslabs < 1 || p->npz / nslabs < 4) throw std::invalid_argument("each slab needs at least 4 planes");
        auto m = new r3d_mesh();
        try {
            m->p = *p;
            m->device = p->gpu_id;
            DeviceGuard dg(m->device);
            cuda_ok(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking), "cudaStreamCreate");
            const int base = p->npz / nslabs, extra = p->npz % nslabs;
            int z0 = 0;
            for (int r = 0; r < nslabs; ++r) {
                const int n = base + (r < extra ? 1 : 0);
                m->slabs.push_back(create_handle(*p, z0, n, m->stream));
                z0 += n;
            }
            std::vector<r3dk::Scalars*> h;
            for (r3d_gpu* g : m->slabs) h.push_back(g->dsc);
            cuda_ok(cudaMalloc(&m->dsc, h.size() * sizeof(r3dk::Scalars*)), "cudaMalloc");
            cuda_ok(cudaMemcpy(m->dsc, h.data(), h.size() * sizeof(r3dk::Scalars*), cudaMemcpyHostToDevice), "copy");
        } catch (...) {
            mesh_free(m);
            throw;
        }
        *out = m;
    });
}

int r3d_mesh_slab(const r3d_mesh* m, int r, int* z0, int* nz) {
    if (!m || r < 0 || r >= (int)m->slabs.size()) return R3D_EINVAL;
    if (z0) *z0 = m->slabs[r]->z0;
    if (nz) *nz = m->slabs[r]->nloc;
    return R3D_OK;
}

int r3d_mesh_upload(r3d_mesh* m, const r3d_host_state* st, const r3d_scalars* sc) {
    return guarded([&] {
        if (!m || !st || !sc) throw std::invalid_argument("null argument");
        for (r3d_gpu* g : m->slabs) {
            r3d_host_state v = slab_view(st, g);
            const int rc = r3d_gpu_upload(g, &v, sc);
            if (rc != R3D_OK) throw Error(rc, r3d_last_error());
        }
    });
}

int r3d_mesh_step(r3d_mesh* m, int nstages, r3d_scalars* sc) {
    return guarded([&] {
        if (!m) throw std::invalid_argument("null handle");
        if (nstages < 1 || nstages > 3) throw std::invalid_argument("nstages must be 1..3");
        if (m->p.tc != 0.0 && m->p.tp != 0.0) throw Error(R3D_EINVAL, "the mesh form needs tc == 0");
        DeviceGuard dg(m->device);
        mesh_step(m, nstages);
        pull_scalars(m->slabs[0], sc);
    });
}

int r3d_mesh_run(r3d_mesh* m, int nsteps, r3d_scalars* sc) {
    return guarded([&] {
        if (!m) throw std::invalid_argument("null handle");
        if (nsteps < 0) throw std::invalid_argument("nsteps < 0");
        if (m->p.tc != 0.0 && m->p.tp != 0.0) throw Error(R3D_EINVAL, "the mesh form needs tc == 0");
        DeviceGuard dg(m->device);
        for (int n = 0; n < nsteps; ++n) mesh_step(m, 3);
        for (r3d_gpu* g : m->slabs) pull_scalars(g, nullptr);  // error flags of every slab
        pull_scalars(m->slabs[0], sc);
    });
}

int r3d_mesh_download(r3d_mesh* m, r3d_host_state* st, r3d_scalars* sc) {
    return guarded([&] {
        if (!m || !st) throw std::invalid_argument("null argument");
        for (r3d_gpu* g : m->slabs) {
            r3d_host_state v = slab_view(st, g);
            const int rc = r3d_gpu_download(g, &v, g == m->slabs.front() ? sc : nullptr);
            if (rc != R3D_OK) throw Error(rc, r3d_last_error());
        }
    });
}

int r3d_mesh_debug_dt_filter(r3d_mesh* m, double margin, int* refolds) {
    if (!m) return R3D_EINVAL;
    int total = 0;
    for (r3d_gpu* g : m->slabs) {
        int n = 0;
        const int rc = r3d_gpu_debug_dt_filter(g, margin, refolds ? &n : nullptr);
        if (rc != R3D_OK) return rc;
        total += n;
    }
    if (refolds) *refolds = total;
    return R3D_OK;
}

int r3d_mesh_destroy(r3d_mesh* m) {
    if (!m) return R3D_OK;
    DeviceGuard dg(m->device);
    cudaStreamSynchronize(m->stream);
    mesh_free(m);
    return R3D_OK;
}

}  // extern "C"
