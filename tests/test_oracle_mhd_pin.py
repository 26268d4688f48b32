"""The oracle's MHD (LMAG) FLUXES against the reference's own Fortran, bit for bit.

tests/golden/mhd_lmag_golden.npz holds FU FV FW FT WW1 WW2 WW3 produced by executing the
`IF (LMAG) THEN` block of golden/fortran/3dmhdsub.f (lines 2146-2651) statement by statement
(oracle/fortran_lmag.py; generator tests/golden/make_mhd_golden.py) on seeded states.  The
oracle's C restatement must reproduce them exactly; where the reference tree is present the
Fortran is executed again here and compared with the fixture.
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import make_mhd_golden as G  # noqa: E402

FIXTURE = os.path.join(HERE, "golden", "mhd_lmag_golden.npz")
ORA = {"FU": "fu", "FV": "fv", "FW": "fw", "FT": "ft", "WW1": "ww1", "WW2": "ww2", "WW3": "ww3"}
INNER = (slice(1, -1), slice(1, -1), slice(1, -1))


@pytest.mark.parametrize("case", sorted(G.CASES))
def test_oracle_lmag_equals_fortran_fixture(case):
    gold = np.load(FIXTURE)
    flags, seed, steps = G.CASES[case]
    om, _ = G.state_pair(flags, seed, steps)
    om.fluxes()
    for k, o in ORA.items():
        ref = gold[f"{case}/{k}"]
        got = om.field(o)[INNER]
        assert np.array_equal(got, ref), f"{k}: max |diff| {float(np.abs(got - ref).max()):.3e}"
        assert np.abs(ref).max() > 0.0


@pytest.mark.skipif(not os.path.exists(os.path.join(G.REF, "golden", "fortran", "3dmhdsub.f")),
                    reason="the reference's Fortran source is not present")
def test_fixture_is_the_fortran_output():
    block = G.Block(os.path.join(G.REF, "golden", "fortran", "3dmhdsub.f"))
    gold = np.load(FIXTURE)
    flags, seed, steps = G.CASES["layer_12x10x16_seed5_3steps"]
    out = G.fortran_rhs(block, flags, seed, steps)
    for k, v in out.items():
        assert np.array_equal(v, gold[f"layer_12x10x16_seed5_3steps/{k}"]), k


def test_translator_refuses_a_recurrence(tmp_path):
    """A statement reading its target at another index cannot be run as one array statement."""
    src = tmp_path / "t.f"
    src.write_text("\tIF (LMAG) THEN\n\tDO 10 K=2,3\n\tDO 10 J=2,3\n\tDO 10 I=2,3\n"
                   "\tRU(I,J,K)=RU(I-1,J,K)+1.0E00\n10\tCONTINUE\n\tENDIF\n")
    block = G.Block(str(src), 1, 7)
    env = {"RU": np.zeros((4, 4, 4))}
    with pytest.raises(ValueError):
        block.run(env)
