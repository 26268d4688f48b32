"""Golden right-hand sides of the MHD (LMAG) branch of FLUXES, from the reference's own Fortran.

Runs the `IF (LMAG) THEN ... ENDIF` block of golden/fortran/3dmhdsub.f (lines 2146-2651)
statement by statement (oracle/fortran_lmag.py) on seeded states built by the oracle, and writes
FU FV FW FT WW1 WW2 WW3 (interior cells) to tests/golden/mhd_lmag_golden.npz.  The reference
C++ aborts on --lmag and no Fortran compiler exists here, so this is how the oracle's MHD
restatement is pinned to the reference.

    python tests/golden/make_mhd_golden.py [path to the reference tree]
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from fortran_lmag import Block, lmag_inputs  # noqa: E402
from oracle import Oracle  # noqa: E402

# the reference checkout: the first argument when run as a script, else $R3D_REFERENCE (no default)
REF = sys.argv[1] if len(sys.argv) > 1 and __name__ == "__main__" else os.environ.get("R3D_REFERENCE", "")
MAG = ["--lmag", "1", "--beta", "10", "--rm", "1", "--ampb", "0.1", "--bfh", "2", "--bzp", "20"]
CASES = {
    "layer_12x10x16_seed5_3steps": (["--npx", "12", "--npy", "10", "--npz", "16"] + MAG, 5, 3),
    "rotation_9x7x11_seed7_2steps": (["--npx", "9", "--npy", "7", "--npz", "11", "--lrot", "1", "--ry", "2",
                                      "--ang", "0.4"] + MAG, 7, 2),
    "strong_8x8x12_seed11_4steps": (["--npx", "8", "--npy", "8", "--npz", "12", "--lmag", "1", "--beta", "2",
                                     "--rm", "0.5", "--ampb", "0.5", "--bfh", "4", "--bzp", "20",
                                     "--pzp", "0.5", "--sigma", "0.1", "--polys", "1.5"], 11, 4),
}
OUT = ("FU", "FV", "FW", "FT", "WW1", "WW2", "WW3")


def state_pair(flags, seed, steps):
    """(oracle holding the MHD state, oracle holding the same state with B = 0)."""
    om = Oracle(flags).init(seed)
    for _ in range(steps):
        om.step()
    oh = Oracle(flags).init(seed)
    for n in ("ru", "rv", "rw", "ro", "tt"):
        oh.field(n)[...] = om.field(n)
    for n in ("bx", "by", "bz"):
        oh.field(n)[...] = 0.0
    oh.fluxes()
    return om, oh


def fortran_rhs(block, flags, seed, steps):
    om, oh = state_pair(flags, seed, steps)
    env = block.run(lmag_inputs(om, oh))
    inner = (slice(1, -1), slice(1, -1), slice(1, -1))
    return {k: env[k][inner].copy() for k in OUT}


def main():
    if not REF or not os.path.isdir(os.path.join(REF, "golden")):
        sys.exit("usage: make_mhd_golden.py <reference checkout> (or set R3D_REFERENCE)")
    block = Block(os.path.join(REF, "golden", "fortran", "3dmhdsub.f"))
    data = {}
    for name, (flags, seed, steps) in CASES.items():
        for k, v in fortran_rhs(block, flags, seed, steps).items():
            data[f"{name}/{k}"] = v
    np.savez_compressed(os.path.join(HERE, "mhd_lmag_golden.npz"), **data)
    print("wrote", len(data), "arrays")


if __name__ == "__main__":
    main()
