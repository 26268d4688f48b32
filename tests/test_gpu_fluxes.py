"""r3d_gpu_fluxes: the FLUXES entry point (src/fluxes.cpp:44-533; LMAG 3dmhdsub.f:2146-2650)
against the oracle's FLUXES of the same state, bit for bit.

The reference checks one FLUXES call against the golden flux1 dump (tests/fluxes_test.cpp:26-55)
and a uniform state for zero fluxes except FW = g*rho (:57-81).  Compared here: every interior
cell of FR and of the B fluxes, and the momentum and energy right-hand sides away from the
domain's top and bottom planes (BCON overwrites those values; the entry point returns 0 there).
"""
import numpy as np
import pytest

import r3d_b200 as R
from oracle import Oracle

MAG = ["--lmag", "1", "--beta", "10", "--rm", "1", "--ampb", "0.1", "--bfh", "2", "--bzp", "20"]
ORA = {"fu": "fu", "fv": "fv", "fw": "fw", "fr": "fr", "ft": "ft", "w1": "ww1", "w2": "ww2", "w3": "ww3"}
CASES = [
    ("hydro", ["--npx", "24", "--npy", "20", "--npz", "32"], 2),
    ("hydro_rot_kappa", ["--npx", "20", "--npy", "16", "--npz", "24", "--lrot", "1", "--ry", "2", "--ang", "0.4",
                         "--pzp", "0.5", "--sigma", "0.1", "--polys", "1.5"], 3),
    ("mhd", ["--npx", "24", "--npy", "20", "--npz", "32"] + MAG, 2),
]


@pytest.mark.gpu
@pytest.mark.parametrize("name,flags,steps", CASES, ids=[c[0] for c in CASES])
def test_fluxes_entry_bitexact(name, flags, steps):
    p = R.parse(flags + ["--seed", "6"])
    st = R.HostState.setup(p)
    with R.GpuSim(p) as sim:
        sim.upload(st)
        sim.run(steps)
        before = st.copy()
        sim.download(before)
        F = sim.fluxes()
        after = st.copy()
        sim.download(after)
    for n in before.fields:  # the call leaves the state as it was
        assert np.array_equal(before.fields[n], after.fields[n]), n
    o = Oracle(flags).init(6)
    for _ in range(steps):
        o.step()
    o.fluxes()
    for n, f in F.items():
        ref = o.field(ORA[n])
        edge_free = n in ("fu", "fv", "fw", "ft")
        ks = slice(2, -2) if edge_free else slice(1, -1)
        a, b = f[ks, 1:-1, 1:-1], ref[ks, 1:-1, 1:-1]
        assert np.array_equal(a, b), f"{n}: max |diff| {float(np.abs(a - b).max()):.3e}"
        if edge_free:
            assert not f[1].any() and not f[-2].any()


@pytest.mark.gpu
def test_fluxes_uniform_state():
    """tests/fluxes_test.cpp:57-81: a state at rest with uniform rho and T has zero fluxes except
    FW = grav * rho."""
    p = R.parse(["--npx", "16", "--npy", "16", "--npz", "16", "--ampt", "0", "--grav", "0.625"])
    st = R.HostState.setup(p)
    for n in st.fields:
        st.fields[n][...] = 0.0
    st.fields["ro"][...] = 1.5
    st.fields["tt"][...] = 2.0
    with R.GpuSim(p) as sim:
        sim.upload(st)
        F = sim.fluxes()
    inner = (slice(2, -2), slice(1, -1), slice(1, -1))
    for n in ("fu", "fv", "fr", "ft"):
        assert not F[n][inner].any(), n
    assert np.all(F["fw"][inner] == 0.625 * 1.5)


@pytest.mark.gpu
@pytest.mark.parametrize("name,flags,steps", [CASES[0], CASES[2]], ids=["hydro", "mhd"])
def test_download_work_is_the_last_third_stage(name, flags, steps):
    """r3d_gpu_download_work after `steps` full steps: uu vv ww of the third stage's input on
    every cell and its right-hand sides (the oracle's arrays after the same steps, which keep
    the last FLUXES call's); the state is unchanged and stepping on stays bit-exact."""
    p = R.parse(flags + ["--seed", "6"])
    st = R.HostState.setup(p)
    o = Oracle(flags).init(6)
    with R.GpuSim(p) as sim:
        sim.upload(st)
        with pytest.raises(R.R3dError) as e:
            sim.work()
        assert e.value.code == R.R3D_ESTATE  # no step yet
        sim.run(steps)
        W = sim.work()
        W2 = sim.work()
        for _ in range(steps):
            o.step()
        for n in ("uu", "vv", "ww"):
            assert np.array_equal(W[n], o.field(n)), n
        for n in ("fu", "fv", "fw", "fr", "ft"):
            ks = slice(2, -2) if n != "fr" else slice(1, -1)
            assert np.array_equal(W[n][ks, 1:-1, 1:-1], o.field(n)[ks, 1:-1, 1:-1]), n
            assert np.array_equal(W[n], W2[n]), n
        sim.step(3)
        o.step()
        after = st.copy()
        sim.download(after)
        for n in ("ru", "rv", "rw", "ro", "tt"):
            assert np.array_equal(after.fields[n][1:-1, 1:-1, 1:-1], o.field(n)[1:-1, 1:-1, 1:-1]), n
        sim.step(2)  # a partial step leaves no third stage
        with pytest.raises(R.R3dError) as e:
            sim.work()
        assert e.value.code == R.R3D_ESTATE


@pytest.mark.gpu
def test_download_work_with_density_diffusion():
    """With ID the velocities are available and the right-hand sides refused."""
    p = R.parse(["--npx", "16", "--npy", "12", "--npz", "20", "--ngrid", "0", "--id", "1", "--dh", "0.5",
                 "--seed", "4"])
    st = R.HostState.setup(p)
    with R.GpuSim(p) as sim:
        sim.upload(st)
        sim.run(2)
        W = sim.work(fluxes=False)
        assert sorted(W) == ["uu", "vv", "ww"] and np.abs(W["uu"]).max() > 0
        with pytest.raises(R.R3dError) as e:
            sim.work()
        assert e.value.code == R.R3D_EINVAL
