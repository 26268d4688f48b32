"""FP64 MHD GPU step vs the oracle's MHD restatement, bit for bit.

The reference C++ aborts on --lmag in FLUXES (src/fluxes.cpp:539-541); the oracle restates the
Fortran LMAG branch (golden/fortran/3dmhdsub.f:2146-2650) on top of the pinned C++ hydro, with
the B stage updates of 3dmhdsub.f:907-1177, Bz = 0 at the top and bottom (src/bcon.cpp:95-98,
136-139) and the magnetic dt terms of src/step.cpp:144-156,195,213-229.  Its MHD initial
condition is pinned to the reference build (tests/test_oracle_ref.py) and its LMAG fluxes to the
reference's Fortran source executed statement by statement (tests/test_oracle_mhd_pin.py), so
GPU == restatement is GPU == reference.
"""
import numpy as np
import pytest

import r3d_b200 as R
from oracle import Oracle, interior

MAG = ["--lmag", "1", "--beta", "10", "--rm", "1", "--ampb", "0.1", "--bfh", "2", "--bzp", "20"]
FIELDS = ["ru", "rv", "rw", "ro", "tt", "bx", "by", "bz"]

CASES = [
    ("mhd_24x20x40", ["--npx", "24", "--npy", "20", "--npz", "40"] + MAG, 7, 5),
    ("mhd_ragged_37x13x23", ["--npx", "37", "--npy", "13", "--npz", "23"] + MAG, 3, 3),
    ("mhd_rotation_kappa", ["--npx", "20", "--npy", "16", "--npz", "32", "--lrot", "1", "--ry", "2",
                            "--ang", "0.4", "--pzp", "0.5", "--sigma", "0.1", "--polys", "1.5"] + MAG, 5, 3),
    ("mhd_strong_field", ["--npx", "16", "--npy", "16", "--npz", "32", "--lmag", "1", "--beta", "2",
                          "--rm", "0.5", "--ampb", "0.5", "--bfh", "4", "--bzp", "20"], 11, 4),
]


def gpu_run(flags, seed, steps, last=3):
    p = R.parse(flags + ["--seed", str(seed)])
    st = R.HostState.setup(p)
    with R.GpuSim(p) as sim:
        sim.upload(st)
        sc = None
        for n in range(steps):
            sc = sim.step(3 if n < steps - 1 else last)
        sim.download(st)
    return st, sc


def check(flags, seed, steps, last=3):
    st, sc = gpu_run(flags, seed, steps, last)
    o = Oracle(flags).init(seed)
    for n in range(steps):
        o.step(3 if n < steps - 1 else last)
    for n in FIELDS:
        d = float(np.abs(interior(st.fields[n]) - interior(o.field(n))).max())
        assert d == 0.0, f"{n}: max |gpu - oracle| = {d:.3e}"
    osc = o.scalars()
    for k in ("dt", "timc", "umach"):
        assert sc[k] == osc[k], k
    assert float(np.abs(interior(st.fields["by"])).max()) > 0.0  # the induction term did act


@pytest.mark.gpu
@pytest.mark.parametrize("name,flags,seed,steps", CASES, ids=[c[0] for c in CASES])
def test_mhd_steps_bitexact(name, flags, seed, steps):
    check(flags, seed, steps)


@pytest.mark.gpu
@pytest.mark.parametrize("stages", [1, 2])
def test_mhd_partial_step_bitexact(stages):
    check(["--npx", "24", "--npy", "20", "--npz", "40"] + MAG, 7, 2, last=stages)


@pytest.mark.gpu
def test_mhd_config2_grid_three_steps():
    """The MHD benchmark grid 126x126x256 (--beta 10 --rm 1, layer ampb 0.1 bfh 2 bzp 20, seed 7)."""
    check(["--npx", "126", "--npy", "126", "--npz", "256"] + MAG, 7, 3)


@pytest.mark.gpu
def test_mhd_config2_hundred_steps():
    """The MHD benchmark case as stated: 126x126x256, --lmag 1 --beta 10 --rm 1, layer
    ampb 0.1 bfh 2 bzp 20, seed 7, 100 RK3 steps, bit for bit (about 45 s of oracle time)."""
    check(["--npx", "126", "--npy", "126", "--npz", "256"] + MAG, 7, 100)


@pytest.mark.gpu
def test_mhd_tile_heights_agree():
    """126x126x64 with MHD takes 32x6 column tiles on one handle and 32x8 on the two slabs of a
    mesh (each too small for two CTAs per SM): the states are bit-identical, and so is the
    oracle's.  The adjoint's recompute on the 32x6 handle reproduces the recorded trajectory
    (a mismatch would raise)."""
    flags = ["--npx", "126", "--npy", "126", "--npz", "64"] + MAG
    p = R.parse(flags + ["--seed", "7"])
    a, sa = gpu_run(flags, 7, 2)
    b = R.HostState.setup(p)
    with R.GpuMesh(p, 2) as m:
        m.upload(b)
        sb = None
        for _ in range(2):
            sb = m.step()
        m.download(b)
    o = Oracle(flags).init(7)
    o.step()
    o.step()
    for n in FIELDS:
        assert np.array_equal(interior(a.fields[n]), interior(b.fields[n])), n
        assert np.array_equal(interior(a.fields[n]), interior(o.field(n))), n
    assert sa["dt"] == sb["dt"] == o.scalars()["dt"]
    st = R.HostState.setup(p)
    with R.GpuSim(p) as sim:
        sim.upload(st)
        sim.adjoint_record(2, 1)
        g = sim.adjoint_backward({n: np.ones_like(x) for n, x in st.fields.items()})
    assert all(np.isfinite(v).all() for v in g.values())
