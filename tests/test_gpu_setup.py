"""The initial state built on the device (r3d_gpu_setup) against the host set-up.

r3d_gpu_setup replaces r3d_setup_host + r3d_gpu_upload (src/main.cpp:134-154,
src/static_ic.cpp:24-161): the metric lines, static columns and magnetic layer come from the
host (1D), kernels fill the fields, and the seeded temperature perturbation - one sequential
RAN2 chain - is drawn on the host plane by plane and applied on the device.  The host set-up is
itself pinned to the compiled reference (test_host.py), so the device state must equal it bit
for bit: every cell of every field, ghosts included, the scalars, and the steps that follow.
"""
import numpy as np
import pytest

import r3d_b200 as R

MAG = ["--lmag", "1", "--beta", "10", "--rm", "1", "--ampb", "0.1", "--bfh", "2", "--bzp", "20"]
CASES = [
    ("config1_32x32x64", ["--npx", "32", "--npy", "32", "--npz", "64", "--seed", "1"], None),
    ("ragged_37x13x23", ["--npx", "37", "--npy", "13", "--npz", "23", "--seed", "5"], None),
    ("mhd_24x20x40", ["--npx", "24", "--npy", "20", "--npz", "40", "--seed", "7"] + MAG, None),
    ("variable_kappa", ["--npx", "24", "--npy", "20", "--npz", "36", "--pzp", "0.5", "--sigma", "0.1",
                        "--polys", "1.5", "--seed", "7"], None),
    ("no_perturbation", ["--npx", "16", "--npy", "12", "--npz", "20", "--ampt", "0"], None),
    ("slab_middle", ["--npx", "24", "--npy", "16", "--npz", "48", "--seed", "3"], (16, 20)),
    ("slab_bottom_mhd", ["--npx", "16", "--npy", "16", "--npz", "40", "--seed", "7"] + MAG, (24, 16)),
    ("fp32bulk", ["--npx", "40", "--npy", "24", "--npz", "32", "--seed", "4", "--precision", "fp32bulk"], None),
]


def _host_state(p, slab):
    return R.HostState.setup(p) if slab is None else R.HostState.setup_slab(p, *slab)


@pytest.mark.gpu
@pytest.mark.parametrize("name,flags,slab", CASES, ids=[c[0] for c in CASES])
def test_device_setup_equals_host_setup(name, flags, slab):
    p = R.parse(flags)
    host = _host_state(p, slab)
    names = list(host.fields)
    out = {}
    for how in ("host", "device"):
        with R.GpuSim(p, slab=slab) as sim:
            if how == "host":
                sim.upload(host)
                sc0 = dict(host.scalars)
            else:
                sc0 = sim.setup()
            st = R.HostState.empty(p) if slab is None else R.HostState({n: np.zeros_like(a) for n, a in host.fields.items()},
                                                                       host.lines, dict(host.scalars))
            sim.download(st)
            first = {n: st.fields[n].copy() for n in names}
            scs = [sim.step() for _ in range(2)] if slab is None else []
            sim.download(st)
            out[how] = (sc0, first, scs, {n: st.fields[n].copy() for n in names})
    (hsc, hfirst, hsteps, hlast), (dsc, dfirst, dsteps, dlast) = out["host"], out["device"]
    assert dsc["tb"] == hsc["tb"] and dsc["nit"] == 0 and dsc["dt"] == 0.0
    for n in names:
        assert np.array_equal(dfirst[n], hfirst[n]), f"{n}: max |device - host| = {np.abs(dfirst[n] - hfirst[n]).max():.3e}"
        assert np.array_equal(dlast[n], hlast[n]), n
    assert dsteps == hsteps


@pytest.mark.gpu
def test_device_setup_of_the_plume_grid_504x504x2048():
    """The FP32-bulk benchmark grid needs 21 GB of host arrays for the host set-up; the device
    set-up needs none.  Spot check against the host set-up on a slab of the same domain (the
    draws of the 1536 planes above it are skipped, as by the host)."""
    flags = ["--npx", "504", "--npy", "504", "--npz", "2048", "--seed", "11", "--tp", "2", "--tc", "0",
             "--xp", "10", "--yp", "10", "--zp", "0", "--hh", "1"]
    p = R.parse(flags)
    with R.GpuSim(p) as sim:
        sc = sim.setup()
        m, e = sim.totals()
        st = sim.step()
    assert np.isfinite(m) and np.isfinite(e) and st["dt"] > 0 and sc["nit"] == 0
    slab = (1536, 64)
    host = R.HostState.setup_slab(p, *slab)
    with R.GpuSim(p, slab=slab) as sim:
        sim.setup()
        got = R.HostState({n: np.zeros_like(a) for n, a in host.fields.items()}, host.lines, dict(host.scalars))
        sim.download(got)
    for n in host.fields:
        assert np.array_equal(got.fields[n], host.fields[n]), n
