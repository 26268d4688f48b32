"""The third stage's filtered dt fold on the GPU: the dt is the same bit for bit whether the
filter skips cells, every step fails its check and re-evaluates the limits, or the handle is a
z slab (exact running bounds only).

The reference evaluates every cell's limits (src/step.cpp:122-229); the filter only decides
which cells cannot change the minimum, and the check in step_end makes the skipped set
provably irrelevant or triggers the full evaluation.
"""
import numpy as np
import pytest

import r3d_b200 as R
from oracle import Oracle, interior

HYDRO = ["--npx", "32", "--npy", "32", "--npz", "64"]
MAG = ["--lmag", "1", "--beta", "10", "--rm", "1", "--ampb", "0.1", "--bfh", "2", "--bzp", "20"]
FIELDS = ["ru", "rv", "rw", "ro", "tt", "bx", "by", "bz"]


def run(flags, seed, steps, margin=None):
    p = R.parse(flags + ["--seed", str(seed)])
    st = R.HostState.setup(p)
    with R.GpuSim(p) as sim:
        if margin is not None:
            sim.debug_dt_filter(margin)
        sim.upload(st)
        dts = []
        for _ in range(steps):
            dts.append(sim.step()["dt"])
        refolds = sim.debug_dt_filter()
        sim.download(st)
    return st, dts, refolds


@pytest.mark.gpu
@pytest.mark.parametrize("name,flags,seed,steps", [
    ("hydro_config1", HYDRO, 1, 20),
    ("mhd", ["--npx", "24", "--npy", "20", "--npz", "40"] + MAG, 7, 6),
    ("variable_kappa", ["--npx", "24", "--npy", "20", "--npz", "36", "--pzp", "0.5", "--sigma", "0.1",
                        "--polys", "1.5"], 7, 6),
])
def test_forced_refold_is_bitexact_with_oracle(name, flags, seed, steps):
    """A negative margin puts every threshold on the wrong side: each step's check fails and
    the limits are evaluated again over the whole state.  State and dt stay the oracle's."""
    st, dts, refolds = run(flags, seed, steps, margin=-0.5)
    assert refolds == steps
    o = Oracle(flags).init(seed)
    odts = []
    for _ in range(steps):
        o.step(3)
        odts.append(o.scalars()["dt"])
    assert dts == odts
    for n in FIELDS[: 8 if "--lmag" in flags else 5]:
        assert np.array_equal(interior(st.fields[n]), interior(o.field(n))), n


@pytest.mark.gpu
def test_default_margin_rarely_refolds_and_matches_no_threshold():
    """The default margin leaves the check satisfied in nearly every step; a huge margin (no
    threshold skipping) gives the identical dt sequence."""
    flags = ["--npx", "64", "--npy", "48", "--npz", "96"]
    a, da, ra = run(flags, 3, 30)
    b, db, rb = run(flags, 3, 30, margin=1e30)
    assert da == db
    assert rb == 0
    assert ra <= 3, f"{ra} refolds in 30 steps"
    for n in FIELDS[:5]:
        assert np.array_equal(interior(a.fields[n]), interior(b.fields[n])), n


@pytest.mark.gpu
def test_fp32bulk_forced_refold_identical():
    """FP32-bulk: the filtered fold, the forced re-evaluation and the threshold-free fold give
    the same dt sequence and state bit for bit."""
    flags = ["--npx", "48", "--npy", "40", "--npz", "64", "--precision", "fp32bulk"]
    a, da, ra = run(flags, 5, 12)
    b, db, rb = run(flags, 5, 12, margin=-0.5)
    c, dc, rc = run(flags, 5, 12, margin=1e30)
    assert rb == 12 and rc == 0
    assert da == db == dc
    for n in FIELDS[:5]:
        assert np.array_equal(a.fields[n], b.fields[n]), n
        assert np.array_equal(a.fields[n], c.fields[n]), n


@pytest.mark.gpu
@pytest.mark.parametrize("margin", [None, -0.5])
def test_slabs_filter_on_their_own_limits(margin):
    """z slabs take their thresholds from their own limits and check their own folds: with
    the default margin (rare refolds) and with a negative one (every slab refolds every step)
    the mesh reproduces the single domain bit for bit."""
    flags = ["--npx", "40", "--npy", "24", "--npz", "48", "--seed", "9"]
    p = R.parse(flags)
    ref, dts, _ = run(flags[:-2], 9, 6)
    st = R.HostState.setup(p)
    with R.GpuMesh(p, 3) as m:
        if margin is not None:
            m.debug_dt_filter(margin)
        m.upload(st)
        got = [m.step()["dt"] for _ in range(6)]
        refolds = m.debug_dt_filter()
        m.download(st)
    assert got == dts
    for n in FIELDS[:5]:
        assert np.array_equal(interior(st.fields[n]), interior(ref.fields[n])), n
    if margin is not None:
        assert refolds == 6 * 3
    else:
        assert refolds <= 3
