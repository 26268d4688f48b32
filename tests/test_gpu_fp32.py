"""FP32-bulk form against the FP64 form (which is bit-exact with the reference).

The FP32-bulk state stores momenta and the deviations of rho and T from the static polytrope
in FP32 and evaluates the stencils in FP32; background parts of the z terms, the stage
accumulation arithmetic, BCON, the dt reduction and the time sum stay in FP64.  Bar: per-field
relative L2 error <= 1e-5 after 100 steps (measured ~3e-7 for the momenta, ~1e-11 for rho,
~3e-10 for T), relative L-infinity <= 1e-4, and total mass / energy drift equal to the FP64
run's to within 1e-9 relative of the totals.
"""
import numpy as np
import pytest

import r3d_b200 as R

FIELDS = ["ru", "rv", "rw", "ro", "tt"]


def run(flags, prec, steps):
    p = R.parse(flags + ["--precision", prec])
    st = R.HostState.setup(p)
    with R.GpuSim(p) as sim:
        sim.upload(st)
        m0, e0 = sim.totals()
        sc = sim.run(steps)
        m1, e1 = sim.totals()
        sim.download(st)
    return st, sc, (m0, e0, m1, e1)


@pytest.mark.gpu
@pytest.mark.parametrize("flags,steps", [
    (["--npx", "64", "--npy", "64", "--npz", "128", "--seed", "3"], 100),
    (["--npx", "37", "--npy", "29", "--npz", "45", "--seed", "5", "--ngrid", "2", "--izcon", "1"], 60),
    (["--npx", "40", "--npy", "24", "--npz", "64", "--seed", "7", "--pzp", "0.5", "--sigma", "0.1",
      "--polys", "1.5", "--lrot", "1", "--ry", "2", "--ang", "0.3"], 60),
])
def test_fp32bulk_error_vs_fp64(flags, steps):
    a, sa, ta = run(flags, "fp64", steps)
    b, sb, tb = run(flags, "fp32bulk", steps)
    for n in FIELDS:
        x, y = a.fields[n][1:-1, 1:-1, 1:-1], b.fields[n][1:-1, 1:-1, 1:-1]
        l2 = np.linalg.norm(x - y) / np.linalg.norm(x)
        li = np.abs(x - y).max() / np.abs(x).max()
        assert l2 <= 1e-5, f"{n}: relative L2 {l2:.3e}"
        assert li <= 1e-4, f"{n}: relative Linf {li:.3e}"
    assert abs(sa["timc"] - sb["timc"]) <= 1e-6 * sa["timc"]
    assert sa["nit"] == sb["nit"] == steps
    for q in (0, 1):  # drift of mass, energy
        da = (ta[q + 2] - ta[q]) / abs(ta[q])
        db = (tb[q + 2] - tb[q]) / abs(tb[q])
        assert abs(da - db) <= 1e-9, (q, da, db)


@pytest.mark.gpu
def test_fp32bulk_upload_download_roundtrip_and_determinism():
    flags = ["--npx", "24", "--npy", "16", "--npz", "32", "--seed", "2", "--precision", "fp32bulk"]
    p = R.parse(flags)
    st = R.HostState.setup(p)
    ref = st.copy()
    with R.GpuSim(p) as sim:
        sim.upload(st)
        sim.download(st)
        for n in FIELDS:  # deviations round to float once: relative error <= 2^-24 of |value|
            d = np.abs(st.fields[n] - ref.fields[n])[1:-1, 1:-1, 1:-1]
            assert (d <= 6e-8 * np.abs(ref.fields[n][1:-1, 1:-1, 1:-1]) + 1e-30).all(), n
        sim.upload(ref)
        s1 = sim.run(5)
        o1 = R.HostState.empty(p)
        sim.download(o1)
        sim.upload(ref)
        s2 = sim.run(5)
        o2 = R.HostState.empty(p)
        sim.download(o2)
    assert s1 == s2
    for n in FIELDS:
        assert np.array_equal(o1.fields[n], o2.fields[n]), n


@pytest.mark.gpu
def test_device_compare_equals_host_norms():
    """r3d_gpu_compare (the on-device error norms the large-grid checks use) against numpy on
    the downloaded states: FP32-bulk vs FP64 and FP64 vs FP64 after a few steps."""
    flags = ["--npx", "40", "--npy", "24", "--npz", "32", "--seed", "4"]
    p64, p32 = R.parse(flags), R.parse(flags + ["--precision", "fp32bulk"])
    st = R.HostState.setup(p64)
    with R.GpuSim(p64) as a, R.GpuSim(p32) as b, R.GpuSim(p64) as c:
        for sim, n in ((a, 5), (b, 5), (c, 4)):
            sim.upload(st)
            sim.run(n)
        got = {"fp32": b.compare(a), "fp64": c.compare(a)}
        host = {}
        for k, sim in (("a", a), ("b", b), ("c", c)):
            h = R.HostState.empty(p64)
            sim.download(h)
            host[k] = h
    for key, other in (("fp32", "b"), ("fp64", "c")):
        for n in FIELDS:
            x = host["a"].fields[n][1:-1, 1:-1, 1:-1]
            y = host[other].fields[n][1:-1, 1:-1, 1:-1]
            l2 = np.linalg.norm(y - x) / np.linalg.norm(x)
            li = np.abs(y - x).max() / np.abs(x).max()
            assert got[key][n]["rel_l2"] == pytest.approx(l2, rel=1e-9, abs=1e-300), (key, n)
            assert got[key][n]["rel_linf"] == pytest.approx(li, rel=1e-12, abs=1e-300), (key, n)
    assert all(v["rel_l2"] > 0 for v in got["fp64"].values())  # one step apart: not identical


@pytest.mark.gpu
def test_plume_504x504x2048_fp32bulk_vs_fp64():
    """The FP32-bulk benchmark configuration: 504 x 504 x 2048 with the reference's plume top
    boundary (tp 2, itcon 1, Gaussian at xp = yp = 10, zp 0, hh 1; src/bcon.cpp:43-70), seed 11,
    50 steps, the FP64 form alongside from the same initial state (63 + 32 GB on the device, built
    there by r3d_gpu_setup).
    Errors are computed on the device; bar as above: rel L2 <= 1e-5, rel Linf <= 1e-4 per field,
    equal drift of mass and energy, and the FP32-bulk step faster."""
    flags = ["--npx", "504", "--npy", "504", "--npz", "2048", "--seed", "11", "--tp", "2", "--tc", "0",
             "--xp", "10", "--yp", "10", "--zp", "0", "--hh", "1"]
    p64, p32 = R.parse(flags), R.parse(flags + ["--precision", "fp32bulk"])
    drift, ms = {}, {}
    with R.GpuSim(p64) as a, R.GpuSim(p32) as b:
        for k, sim in (("fp64", a), ("fp32", b)):
            sim.setup()  # the initial state built on the device: no 21 GB host copy
            m0, e0 = sim.totals()
            sc, tm = sim.run_timed(50)
            m1, e1 = sim.totals()
            drift[k] = ((m1 - m0) / m0, (e1 - e0) / e0)
            ms[k] = tm["total_ms"] / 50
            assert sc["nit"] == 50
        err = b.compare(a)
    for n in FIELDS:
        assert err[n]["rel_l2"] <= 1e-5, (n, err[n])
        assert err[n]["rel_linf"] <= 1e-4, (n, err[n])
    for q in (0, 1):
        assert abs(drift["fp64"][q] - drift["fp32"][q]) <= 1e-9, (q, drift)
    assert ms["fp32"] < ms["fp64"], ms
