"""FP64 GPU step vs the oracle, bit for bit (the reference's own bar: tests/golden_util.hpp:94-104
compares interiors with max |diff| == 0, and tests/gpu_equivalence_test.cpp:143-174 also
requires dt and nit to be equal).

Each case builds the initial state with the product's host set-up (itself checked against the
oracle in test_host.py), steps it on the GPU through the C ABI, and compares the interiors of
ru rv rw ro tt and the scalars with the C restatement stepped from its own initial state.
"""
import numpy as np
import pytest

import r3d_b200 as R
from oracle import Oracle, Reference, interior

PRIMARY = ["ru", "rv", "rw", "ro", "tt"]

# (name, flags, seed, steps)
HYDRO_CASES = [
    ("config1_32x32x64_seed1", ["--npx", "32", "--npy", "32", "--npz", "64"], 1, 20),
    ("golden_16x16x32", ["--npx", "16", "--npy", "16", "--npz", "32"], 62659, 3),
    ("ragged_37x13x23", ["--npx", "37", "--npy", "13", "--npz", "23"], 5, 5),
    ("ngrid2_izcon1_itcon0", ["--npx", "24", "--npy", "20", "--npz", "36", "--ngrid", "2",
                              "--izcon", "1", "--itcon", "0"], 5, 5),
    ("ngrid0_rotation_tc", ["--npx", "24", "--npy", "20", "--npz", "36", "--ngrid", "0",
                            "--lrot", "1", "--ry", "2", "--ang", "0.3", "--tc", "0.5"], 5, 5),
    ("variable_kappa", ["--npx", "24", "--npy", "20", "--npz", "36", "--pzp", "0.5",
                        "--sigma", "0.1", "--polys", "1.5"], 7, 5),
    ("itcon4", ["--npx", "24", "--npy", "16", "--npz", "40", "--itcon", "4"], 3, 4),
    ("no_plume", ["--npx", "24", "--npy", "16", "--npz", "40", "--tp", "0"], 3, 4),
    ("min_size", ["--npx", "3", "--npy", "3", "--npz", "8"], 2, 3),
    # itcon 2: constant top T and the localized embedded heat loss of the Fortran FLUXES
    # (3dmhdsub.f:1799-1822; the oracle's term is pinned to that source, test_oracle_itc2_pin.py)
    ("itcon2_heat_loss", ["--npx", "24", "--npy", "20", "--npz", "36", "--itcon", "2", "--tp", "0.5",
                          "--xp", "8", "--yp", "12", "--zp", "0.1"], 5, 5),
    ("itcon2_ramp_hh07", ["--npx", "21", "--npy", "17", "--npz", "30", "--itcon", "2", "--tp", "0.3",
                          "--tc", "0.002", "--qfh", "0.001", "--hh", "0.7", "--xp", "6", "--yp", "9",
                          "--zp", "0.3"], 7, 6),
    # itcon 3: the top temperature is the stage's own (no BCON rewrite, 3dmhdsub.f:2807-2880), so
    # the top plane's energy flux is formed in full; both conductivity forms, with rotation
    ("itcon3_free_top", ["--npx", "24", "--npy", "20", "--npz", "36", "--itcon", "3", "--tp", "0.5",
                         "--lrot", "1", "--ry", "2", "--ang", "0.3"], 5, 6),
    ("itcon3_variable_kappa_izcon1", ["--npx", "21", "--npy", "17", "--npz", "30", "--itcon", "3",
                                      "--izcon", "1", "--ngrid", "2", "--pzp", "0.5", "--sigma", "0.1",
                                      "--polys", "1.5"], 7, 5),
    # density diffusion (ID 1, 2; 3dmhdsub.f:1316-1386, uniform grid; the oracle's term is pinned
    # to that source, test_oracle_id_pin.py): horizontal, vertical, both with the ID 2 profile,
    # and with a free top temperature on a ragged grid
    ("id1_dh", ["--npx", "24", "--npy", "20", "--npz", "36", "--ngrid", "0", "--id", "1", "--dh", "0.5"], 5, 4),
    ("id1_dv", ["--npx", "24", "--npy", "20", "--npz", "36", "--ngrid", "0", "--id", "1", "--dv", "0.75"], 5, 4),
    ("id2_dh_dv", ["--npx", "24", "--npy", "20", "--npz", "36", "--ngrid", "0", "--id", "2", "--dh", "0.25",
                   "--dv", "0.25", "--zmax", "2"], 7, 4),
    ("id1_itcon3_ragged", ["--npx", "21", "--npy", "17", "--npz", "30", "--ngrid", "0", "--id", "1", "--dh", "0.5",
                           "--dv", "0.5", "--itcon", "3", "--tp", "0.5"], 3, 5),
]


def gpu_run(flags, seed, steps, last_stages=3, use_run=False):
    p = R.parse(flags + ["--seed", str(seed)])
    st = R.HostState.setup(p)
    with R.GpuSim(p) as sim:
        sim.upload(st)
        if use_run and last_stages == 3:
            sc = sim.run(steps)
        else:
            sc = None
            for n in range(steps):
                sc = sim.step(3 if n < steps - 1 else last_stages)
        sim.download(st)
    return st, sc


def oracle_run(flags, seed, steps, last_stages=3):
    o = Oracle(flags).init(seed)
    for n in range(steps):
        o.step(3 if n < steps - 1 else last_stages)
    return o


def assert_bitexact(st, o, sc, names=PRIMARY):
    for n in names:
        a, b = interior(st.fields[n]), interior(o.field(n))
        diff = float(np.abs(a - b).max())
        assert diff == 0.0, f"{n}: max |gpu - oracle| = {diff:.3e}"
        # the x/y ghost images the kernels write (every interior plane, corners included)
        ga, gb = st.fields[n][1:-1], o.field(n)[1:-1]
        assert np.array_equal(ga, gb), f"{n}: ghost images differ"
    osc = o.scalars()
    for k in ("dt", "timc", "timt", "umach"):
        assert sc[k] == osc[k], f"{k}: gpu {sc[k]!r} oracle {osc[k]!r}"
    assert sc["nit"] == int(osc["nit"])


@pytest.mark.gpu
@pytest.mark.parametrize("name,flags,seed,steps", HYDRO_CASES, ids=[c[0] for c in HYDRO_CASES])
def test_hydro_steps_bitexact(name, flags, seed, steps):
    st, sc = gpu_run(flags, seed, steps)
    o = oracle_run(flags, seed, steps)
    assert_bitexact(st, o, sc)


@pytest.mark.gpu
@pytest.mark.parametrize("kchunk", [1, 2, 3, 7])
@pytest.mark.parametrize("name,flags,seed", [
    ("ragged_37x13x23", ["--npx", "37", "--npy", "13", "--npz", "23"], 5),
    ("variable_kappa_itcon3", ["--npx", "24", "--npy", "20", "--npz", "30", "--pzp", "0.5", "--sigma", "0.1",
                               "--polys", "1.5", "--itcon", "3"], 7),
], ids=["ragged", "variable_kappa_itcon3"])
def test_shallow_z_chunks_bitexact(name, flags, seed, kchunk, monkeypatch):
    """Chunks of 1, 2, 3 and 7 planes (R3D_KCHUNK): every chunk starts from its own plane above
    and runs the raw ring's first slots, so the ring's start-up, its refill guards and the
    registers carried from plane to plane are exercised at every depth."""
    monkeypatch.setenv("R3D_KCHUNK", str(kchunk))
    st, sc = gpu_run(flags, seed, 4)
    o = oracle_run(flags, seed, 4)
    assert_bitexact(st, o, sc)


@pytest.mark.gpu
@pytest.mark.parametrize("stages", [1, 2, 3])
def test_partial_step_bitexact(stages):
    """step(nstages) for the per-stage bisection the reference tests use
    (tests/gpu_equivalence_test.cpp:178-332)."""
    flags = ["--npx", "32", "--npy", "24", "--npz", "48"]
    st, sc = gpu_run(flags, 11, 2, last_stages=stages)
    o = oracle_run(flags, 11, 2, last_stages=stages)
    assert_bitexact(st, o, sc)


@pytest.mark.gpu
def test_run_matches_step_loop():
    """r3d_gpu_run (device-resident loop) equals repeated r3d_gpu_step."""
    flags = ["--npx", "40", "--npy", "24", "--npz", "48"]
    a, sa = gpu_run(flags, 9, 6)
    b, sb = gpu_run(flags, 9, 6, use_run=True)
    for n in PRIMARY:
        assert np.array_equal(interior(a.fields[n]), interior(b.fields[n])), n
    assert sa == sb


@pytest.mark.gpu
@pytest.mark.parametrize("flags,lead", [
    (["--npx", "40", "--npy", "24", "--npz", "48"], 1),
    (["--npx", "24", "--npy", "20", "--npz", "40", "--lmag", "1", "--beta", "10", "--rm", "1", "--ampb", "0.1",
      "--bfh", "2", "--bzp", "20"], 2),
    (["--npx", "40", "--npy", "24", "--npz", "48", "--precision", "fp32bulk"], 0),
], ids=["hydro_odd_parity", "mhd_even_parity", "fp32bulk"])
def test_graph_replay_matches_step_loop(flags, lead):
    """r3d_gpu_run replays a captured two-step CUDA graph (per buffer parity); after `lead`
    partial stages and across two run calls it equals the eager step loop bit for bit."""
    p = R.parse(flags + ["--seed", "12"])
    outs = []
    for use_run in (False, True):
        st = R.HostState.setup(p)
        with R.GpuSim(p) as sim:
            sim.upload(st)
            if lead:
                sim.step(lead)
            if use_run:
                sim.run(5)
                sc = sim.run(4)
            else:
                for _ in range(9):
                    sc = sim.step()
            sim.download(st)
        outs.append((st, sc))
    (a, sa), (b, sb) = outs
    for n in a.fields:
        assert np.array_equal(a.fields[n], b.fields[n]), n
    assert sa == sb


@pytest.mark.gpu
def test_graph_replay_survives_reupload_and_enqueue():
    """The captured step graph keeps working after a new upload (same buffers, new contents) and
    through r3d_gpu_enqueue: the result equals a fresh handle's step loop."""
    flags = ["--npx", "40", "--npy", "24", "--npz", "48", "--seed", "4"]
    p = R.parse(flags)
    ref, sref = gpu_run(flags[:-2], 4, 6)
    st = R.HostState.setup(p)
    with R.GpuSim(p) as sim:
        sim.upload(st)
        sim.run(6)                      # captures the graph on other contents
        sim.upload(st)                  # back to the initial state
        sim.enqueue(4)
        sc = sim.run(2)
        sim.download(st)
    for n in PRIMARY:
        assert np.array_equal(interior(st.fields[n]), interior(ref.fields[n])), n
    assert sc == sref


@pytest.mark.gpu
def test_gpu_vs_reference_build_directly():
    """When the reference CPU build is present, also compare against it without the oracle."""
    if not Reference.available():
        pytest.skip("reference build not present")
    flags = ["--npx", "32", "--npy", "32", "--npz", "64"]
    st, sc = gpu_run(flags, 1, 20)
    rf, _, rs, _ = Reference.run(flags + ["--npey", "1"], nranks=2, seed=1, nsteps=20, omp_threads=4)
    for n in PRIMARY:
        assert float(np.abs(interior(st.fields[n]) - interior(rf[n])).max()) == 0.0, n
    for k in ("dt", "timc", "umach"):
        assert sc[k] == rs[k], k


@pytest.mark.gpu
def test_headline_grid_three_steps_bitexact():
    """The 504x504x512 hydro grid (seed 3) the throughput is quoted on: three full RK3 steps
    through the device-resident loop (the graph replay the benchmark uses), state with ghost
    images and scalars bit for bit after each step (about 30 s of oracle time, 20 GB of host
    memory)."""
    flags = ["--npx", "504", "--npy", "504", "--npz", "512"]
    p = R.parse(flags + ["--seed", "3"])
    st = R.HostState.setup(p)
    o = Oracle(flags).init(3)
    with R.GpuSim(p) as sim:
        sim.upload(st)
        for n in range(3):
            sc = sim.run(1)
            o.step()
            sim.download(st)
            assert_bitexact(st, o, sc)
