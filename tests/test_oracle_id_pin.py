"""The oracle's density diffusion (ID 1 and 2) against the reference's own Fortran, bit for bit.

The term exists only in the Fortran FLUXES (golden/fortran/3dmhdsub.f:1316-1386; the reference
C++ aborts on --id, src/fluxes.cpp:46-51).  tests/golden/id_diffusion_golden.npz holds the FR the
block produces from zeros - its ghost-plane mirror and uniform-grid HORIZONTAL_MEAN carried out
as written, its loops executed statement by statement by oracle/fortran_lmag.py (generator
tests/golden/make_id_golden.py) - on states of the oracle after a few steps.  The oracle's C
restatement (the function its FLUXES calls) must reproduce them exactly; where the reference
tree is present the Fortran is executed again and compared with the fixture.
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import make_id_golden as G  # noqa: E402
from oracle import Oracle  # noqa: E402

FIXTURE = os.path.join(HERE, "golden", "id_diffusion_golden.npz")
SRC = os.path.join(G.REF, "golden", "fortran", "3dmhdsub.f")


@pytest.mark.parametrize("case", sorted(G.CASES))
def test_oracle_density_diffusion_equals_fortran_fixture(case):
    gold = np.load(FIXTURE)[case]
    flags, seed, steps = G.CASES[case]
    o = Oracle(flags).init(seed)
    for _ in range(steps):
        o.step()
    got = o.density_diffusion()[1:-1, 1:-1, 1:-1]
    assert np.array_equal(got, gold), f"max |diff| {float(np.abs(got - gold).max()):.3e}"
    assert np.abs(gold).max() > 0.0


@pytest.mark.skipif(not os.path.exists(SRC), reason="the reference's Fortran source is not present")
def test_fixture_is_the_fortran_output():
    blocks = G.source(SRC)
    gold = np.load(FIXTURE)
    for case, (flags, seed, steps) in G.CASES.items():
        _, fr = G.fortran_diffusion(blocks, flags, seed, steps)
        assert np.array_equal(fr[1:-1, 1:-1, 1:-1], gold[case]), case


def test_horizontal_mean_is_the_sequential_sum():
    """HORIZONTAL_MEAN adds the plane's interior values in loop order (j outer, i inner) and
    divides by FLOAT(NPX*NPY): a different order rounds differently."""
    rng = np.random.default_rng(1)
    var = rng.standard_normal((3, 7, 9)) * 1e3 + 1.0
    m = G.horizontal_mean(var, 7, 5)
    for k in range(3):
        s = 0.0
        for v in var[k, 1:-1, 1:-1].ravel():
            s += float(v)
        assert m[k] == s / 35.0


def test_density_diffusion_refusals():
    """The Fortran's HORIZONTAL_MEAN stops on a stretched grid (3dmhdsub.f:3187-3190), so ID
    needs --ngrid 0; ID must be 1 or 2."""
    for flags in (["--id", "1", "--dh", "0.5"], ["--ngrid", "0", "--id", "3", "--dh", "0.5"]):
        o = Oracle(["--npx", "8", "--npy", "8", "--npz", "10"] + flags).init(3)
        with pytest.raises(RuntimeError):
            o.step()
