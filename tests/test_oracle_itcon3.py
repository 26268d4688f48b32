"""itcon 3 in the oracle: the top temperature is left to the stage.

The Fortran BCON (golden/fortran/3dmhdsub.f:2807-2880) rewrites TT on the top plane for ITCON
0, 1, 2 and 4 and has no branch for 3 ("thermal", 3dmhdparam.f:66-67), while its FLUXES forms
FT on every interior plane, the top one included; the reference C++ stops on --itcon 3
(src/fluxes.cpp:50).  So one stage from the same state differs from the itcon-0 stage only in
the top plane's temperature, and that temperature is the stage's own value.
"""
import numpy as np

from oracle import Oracle

FIELDS = ["ru", "rv", "rw", "ro", "tt"]
BASE = ["--npx", "12", "--npy", "10", "--npz", "16", "--tp", "0"]


def _one_stage(itcon, nstages=1):
    o = Oracle(BASE + ["--itcon", str(itcon)]).init(9)
    t0 = o.field("tt").copy()
    o.step(nstages)
    return o, t0


def test_itcon3_differs_from_itcon0_only_in_the_top_temperature():
    a, t0 = _one_stage(0)
    b, _ = _one_stage(3)
    for f in FIELDS:
        fa, fb = a.field(f)[:, 1:-1, 1:-1], b.field(f)[:, 1:-1, 1:-1]
        assert np.array_equal(fa[2:-1], fb[2:-1]), f
        if f != "tt":
            assert np.array_equal(fa[1], fb[1]), f
    top0, top3 = a.field("tt")[1, 1:-1, 1:-1], b.field("tt")[1, 1:-1, 1:-1]
    assert (top0 == 1.0).all()
    assert np.isfinite(top3).all() and not (top3 == t0[1, 1:-1, 1:-1]).all() and not (top3 == 1.0).all()


def test_itcon3_top_temperature_feeds_the_next_stages():
    a, _ = _one_stage(0, 3)
    b, _ = _one_stage(3, 3)
    assert not np.array_equal(a.field("tt")[2, 1:-1, 1:-1], b.field("tt")[2, 1:-1, 1:-1])
