"""z-slab decomposition on the GPU: every slab count reproduces the single-domain run bit for bit.

The reference splits z over npez MPI ranks with a ghost-plane exchange per stage and an
MPI_Allreduce of the dt limits per step (src/communicate.cpp:70-182, src/step.cpp:224).  The
in-process mesh (r3d_mesh_*) runs that exact sequence with several slab handles on one device;
the NCCL transport (r3d_gpu_halo_init) is exercised with a single rank (its collectives run
with nranks = 1: no cross-process waits on one GPU).
"""
import numpy as np
import pytest

import r3d_b200 as R

MAG = ["--lmag", "1", "--beta", "10", "--rm", "1", "--ampb", "0.1", "--bfh", "2", "--bzp", "20"]
CASES = [
    ("hydro", ["--npx", "40", "--npy", "24", "--npz", "32"], (2, 3, 4)),
    ("hydro_ragged_rot_flux", ["--npx", "37", "--npy", "13", "--npz", "23", "--lrot", "1", "--ry", "2",
                               "--ang", "0.4", "--izcon", "1", "--itcon", "0", "--tp", "0"], (2, 5)),
    ("variable_kappa", ["--npx", "24", "--npy", "20", "--npz", "30", "--pzp", "0.5", "--sigma", "0.1",
                        "--polys", "1.5"], (3,)),
    ("itcon3", ["--npx", "24", "--npy", "16", "--npz", "30", "--itcon", "3", "--tp", "0.5"], (2, 3)),
    ("id1_dh_dv", ["--npx", "24", "--npy", "16", "--npz", "30", "--ngrid", "0", "--id", "1", "--dh", "0.5",
                   "--dv", "0.5"], (2, 3)),
    ("mhd", ["--npx", "24", "--npy", "20", "--npz", "40"] + MAG, (2, 3)),
    ("fp32bulk", ["--npx", "40", "--npy", "24", "--npz", "32", "--precision", "fp32bulk"], (2, 4)),
]


def single(p, steps, last=3):
    st = R.HostState.setup(p)
    with R.GpuSim(p) as sim:
        sim.upload(st)
        sc = None
        for n in range(steps):
            sc = sim.step(3 if n < steps - 1 else last)
        sim.download(st)
    return st, sc


def meshed(p, nslabs, steps, last=3):
    st = R.HostState.setup(p)
    with R.GpuMesh(p, nslabs) as m:
        m.upload(st)
        sc = None
        for n in range(steps):
            sc = m.step(3 if n < steps - 1 else last)
        m.download(st)
    return st, sc


def same(a, b):
    for n in a.fields:
        x, y = a.fields[n][1:-1, 1:-1, 1:-1], b.fields[n][1:-1, 1:-1, 1:-1]
        assert np.array_equal(x, y), f"{n}: max |diff| {float(np.abs(x - y).max()):.3e}"


@pytest.mark.gpu
@pytest.mark.parametrize("name,flags,slabs", CASES, ids=[c[0] for c in CASES])
def test_mesh_equals_single_domain(name, flags, slabs):
    p = R.parse(flags + ["--seed", "4"])
    ref, rsc = single(p, 6)
    for s in slabs:
        got, gsc = meshed(p, s, 6)
        same(ref, got)
        for k in ("dt", "timc", "timt", "umach", "nit"):
            assert gsc[k] == rsc[k], (s, k)


@pytest.mark.gpu
@pytest.mark.parametrize("last", [1, 2])
def test_mesh_partial_steps(last):
    p = R.parse(["--npx", "32", "--npy", "16", "--npz", "24", "--seed", "8"])
    ref, rsc = single(p, 3, last)
    got, gsc = meshed(p, 3, 3, last)
    same(ref, got)
    assert gsc["dt"] == rsc["dt"]


@pytest.mark.gpu
def test_slab_handles_single_rank_nccl():
    """One slab covering the domain, joined to a one-rank NCCL exchange."""
    p = R.parse(["--npx", "40", "--npy", "24", "--npz", "32", "--seed", "6"])
    ref, rsc = single(p, 4)
    st = R.HostState.setup_slab(p, 0, p.npz)
    with R.GpuSim(p, slab=(0, p.npz)) as sim:
        sim.halo_init(R.nccl_unique_id(), 0, 1)
        sim.upload(st)
        sc = sim.run(4)
        sim.download(st)
    same(ref, st)
    assert sc["dt"] == rsc["dt"]


@pytest.mark.gpu
def test_slab_errors():
    p = R.parse(["--npx", "16", "--npy", "16", "--npz", "16"])
    with pytest.raises(R.R3dError):
        R.GpuSim(p, slab=(0, 3))          # fewer than 4 planes
    with pytest.raises(R.R3dError):
        R.GpuSim(p, slab=(10, 8))         # beyond the domain
    with pytest.raises(R.R3dError):
        R.GpuMesh(p, 5)                   # 3-plane slabs
    sim = R.GpuSim(p, slab=(4, 8))
    with pytest.raises(R.R3dError):
        sim.halo_init(R.nccl_unique_id(), 0, 2)  # rank 0 must hold the top slab
    st = R.HostState.setup_slab(p, 4, 8)
    sim.upload(st)
    with pytest.raises(R.R3dError):
        sim.adjoint_step({n: np.zeros_like(a) for n, a in st.fields.items()})
    sim.close()
