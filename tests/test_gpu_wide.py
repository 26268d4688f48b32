"""The benchmark's 504 x 504 plane at small depth against the oracle, bit for bit.

504 = 15 x 32 + 24 columns and 63 x 8 rows: partial x tiles, the full y tiling of the benchmark
grid, and a state (8 M cells, 15 arrays) far larger than L2."""
import numpy as np
import pytest

import r3d_b200 as R
from oracle import Oracle, interior


@pytest.mark.gpu
def test_benchmark_plane_two_steps_bitexact():
    flags = ["--npx", "504", "--npy", "504", "--npz", "24"]
    p = R.parse(flags + ["--seed", "3"])
    st = R.HostState.setup(p)
    with R.GpuSim(p) as sim:
        sim.upload(st)
        sim.step()
        sc = sim.step()
        sim.download(st)
    o = Oracle(flags).init(3)
    o.step()
    o.step()
    for n in ("ru", "rv", "rw", "ro", "tt"):
        d = float(np.abs(interior(st.fields[n]) - interior(o.field(n))).max())
        assert d == 0.0, (n, d)
    osc = o.scalars()
    assert sc["dt"] == osc["dt"] and sc["umach"] == osc["umach"]
