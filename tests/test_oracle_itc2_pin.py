"""The oracle's itcon-2 embedded heat loss against the reference's own Fortran, bit for bit.

The term exists only in the Fortran FLUXES (golden/fortran/3dmhdsub.f:1799-1822; the reference
C++ aborts on --itcon 2, src/fluxes.cpp:50).  tests/golden/itc2_heat_golden.npz holds the FT the
block produces, executed statement by statement by oracle/fortran_lmag.py (generator
tests/golden/make_itc2_golden.py), on states of the oracle after a few steps: a steady loss
with HH = 1, and the TANH ramp (TC != 0) with HH != 1.  The oracle's C restatement (the function
its FLUXES calls) must reproduce them exactly; where the reference tree is present the Fortran is
executed again and compared with the fixture.
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import make_itc2_golden as G  # noqa: E402
from oracle import Oracle  # noqa: E402

FIXTURE = os.path.join(HERE, "golden", "itc2_heat_golden.npz")
SRC = os.path.join(G.REF, "golden", "fortran", "3dmhdsub.f")


@pytest.mark.parametrize("case", sorted(G.CASES))
def test_oracle_heat_loss_equals_fortran_fixture(case):
    gold = np.load(FIXTURE)[case]
    flags, seed, steps = G.CASES[case]
    o = Oracle(flags).init(seed)
    for _ in range(steps):
        o.step()
    got = o.heat_loss()[1:-1, 1:-1, 1:-1]
    assert np.array_equal(got, gold), f"max |diff| {float(np.abs(got - gold).max()):.3e}"
    assert np.abs(gold).max() > 0.0 and (gold <= 0.0).all()  # a loss


@pytest.mark.skipif(not os.path.exists(SRC), reason="the reference's Fortran source is not present")
def test_fixture_is_the_fortran_output():
    block = G.Block(SRC, G.FIRST, G.LAST, guard="ITC.EQ.2")
    gold = np.load(FIXTURE)
    for case, (flags, seed, steps) in G.CASES.items():
        _, ft = G.fortran_heat(block, flags, seed, steps)
        assert np.array_equal(ft[1:-1, 1:-1, 1:-1], gold[case]), case


def test_executor_keeps_fortran_single_precision_literals():
    """-4.0E00*LOG(2.0E00) is evaluated in single precision (default REAL), then widened."""
    from fortran_lmag import parse, Block
    b = Block.__new__(Block)
    v = b._value(parse("-4.0E00*LOG(2.0E00)/HH/HH"), {"HH": 0.7}, {})
    expect = float(np.float32(-4.0) * np.float32(np.log(np.float32(2.0)))) / 0.7 / 0.7
    assert v == expect and v != -4.0 * np.log(2.0) / 0.7 / 0.7
