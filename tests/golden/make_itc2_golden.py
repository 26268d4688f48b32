"""Fixture of the itcon-2 embedded heat loss: the reference's Fortran block executed statement by
statement (test infrastructure).

The localized embedded heat loss exists only in the Fortran FLUXES (golden/fortran/3dmhdsub.f,
`IF (ITC.EQ.2) THEN` block, lines 1799-1822); the reference C++ aborts on --itcon 2
(src/fluxes.cpp:50).  oracle/fortran_lmag.py executes the block's source text on the oracle's
state (FT from zeros, RO = 1/rho as at that point of FLUXES, 3dmhdsub.f:1405), for the cases
below, and stores the resulting FT in tests/golden/itc2_heat_golden.npz.

    python tests/golden/make_itc2_golden.py <reference checkout>     (or set R3D_REFERENCE)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from fortran_lmag import Block  # noqa: E402
from oracle import Oracle  # noqa: E402

# the reference checkout: the first argument when run as a script, else $R3D_REFERENCE (no default)
REF = sys.argv[1] if len(sys.argv) > 1 and __name__ == "__main__" else os.environ.get("R3D_REFERENCE", "")
FIRST, LAST = 1799, 1822
CASES = {
    # name: (flags, seed, steps before the evaluation)
    "steady_hh1_12x10x16_seed3_2steps": (["--npx", "12", "--npy", "10", "--npz", "16", "--itcon", "2",
                                          "--tp", "0.5", "--xp", "8", "--yp", "12", "--zp", "0.1"], 3, 2),
    "ramp_hh07_9x11x13_seed5_3steps": (["--npx", "9", "--npy", "11", "--npz", "13", "--itcon", "2", "--tp", "0.3",
                                        "--tc", "0.002", "--qfh", "0.001", "--hh", "0.7", "--xp", "6",
                                        "--yp", "9", "--zp", "0.3"], 5, 3),
}


def fortran_heat(block, flags, seed, steps):
    o = Oracle(flags).init(seed)
    for _ in range(steps):
        o.step()
    sc = o.scalars()
    env = {"FT": np.zeros((o.NZ, o.NY, o.NX)), "RO": 1.0 / o.field("ro")}
    for n in ("exx", "wyy", "zee"):
        env[n.upper()] = np.array(o.line(n))
    p = {k: o.param(k) for k in ("ocv",)}
    env.update(OCV=p["ocv"], TIMT=sc["timi"] + sc["timc"], ITC=2)
    get = dict(zip(flags[::2], flags[1::2]))
    env.update(TP=float(get["--tp"]), TC=float(get.get("--tc", 0.0)), QFH=float(get.get("--qfh", 0.0)),
               HH=float(get.get("--hh", 1.0)), XP=float(get["--xp"]), YP=float(get["--yp"]),
               ZP=float(get["--zp"]))
    env.update(ILAP=2, IX=2, IY=2, NX=o.NX, NY=o.NY, NZ=o.NZ, MYPEZ=0, NPEZ=2)
    block.run(env)
    return o, env["FT"]


def main():
    if not REF or not os.path.isdir(os.path.join(REF, "golden")):
        sys.exit("usage: make_itc2_golden.py <reference checkout> (or set R3D_REFERENCE)")
    block = Block(os.path.join(REF, "golden", "fortran", "3dmhdsub.f"), FIRST, LAST, guard="ITC.EQ.2")
    data = {}
    for name, (flags, seed, steps) in CASES.items():
        _, ft = fortran_heat(block, flags, seed, steps)
        data[name] = ft[1:-1, 1:-1, 1:-1]
    np.savez_compressed(os.path.join(HERE, "itc2_heat_golden.npz"), **data)
    print("wrote", len(data), "arrays")


if __name__ == "__main__":
    main()
