"""Generate tests/golden/reference_pins.json from the reference tree (run where it exists).

Sources, read as text from the reference's own tests (no reference code is executed for these):
  * tests/_ran2_ref.inc        - every 1000th RAN2 draw, seed -62659
  * tests/ran2_ode_test.cpp    - static profile T/R values at NPZ = 32 (golden defaults)
  * tests/params_test.cpp      - widened single-precision defaults, golden Derived constants
Plus runs of the reference CPU sources compiled unmodified (oracle/_ref/libr3dref.so): for a
few hydro configurations, a SHA-256 of each primary field's interior after N steps and the
scalars as hex floats, so the C restatement stays pinned on machines without the reference.

    python tests/golden/make_golden.py [/path/to/reference]
"""
import hashlib
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

# the reference checkout: the first argument, else $R3D_REFERENCE (no default)
REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("R3D_REFERENCE", "")

# hydro configurations recorded from the reference build: (name, flags, seed, nranks, steps)
RUNS = [
    ("config1_32x32x64_seed1_20steps", ["--npx", "32", "--npy", "32", "--npz", "64", "--npey", "1"], 1, 2, 20),
    ("golden_16x16x32_2x2_3steps", ["--npx", "16", "--npy", "16", "--npz", "32", "--npey", "2"], 62659, 4, 3),
    ("ngrid2_izcon1_itcon0_5steps", ["--npx", "24", "--npy", "20", "--npz", "36", "--npey", "1", "--ngrid", "2",
                                     "--izcon", "1", "--itcon", "0"], 5, 2, 5),
    ("rotation_tc_kappa_5steps", ["--npx", "24", "--npy", "20", "--npz", "36", "--npey", "1", "--lrot", "1",
                                  "--ry", "2", "--ang", "0.3", "--tc", "0.5", "--pzp", "0.5", "--sigma", "0.1",
                                  "--polys", "1.5"], 7, 2, 5),
]


def interior_sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a[1:-1, 1:-1, 1:-1], dtype="<f8").tobytes()).hexdigest()


def main():
    if not REF or not os.path.isdir(os.path.join(REF, "tests")):
        sys.exit("usage: make_golden.py <reference checkout> (or set R3D_REFERENCE)")
    pins = {}
    inc = open(os.path.join(REF, "tests", "_ran2_ref.inc")).read()
    pins["ran2_seed62659_every1000"] = [[int(n), float(v)] for n, v in
                                        re.findall(r"\{\s*(\d+)\s*,\s*([0-9.eE+-]+)\s*\}", inc)]
    ode = open(os.path.join(REF, "tests", "ran2_ode_test.cpp")).read()
    prof = {}
    for arr, idx, val in re.findall(r"EXPECT_DOUBLE_EQ\((T|R)\[(\d+)\],\s*([0-9.eE+-]+)\)", ode):
        prof[f"{arr}{idx}"] = float(val)
    pins["static_profile_npz32"] = prof
    par = open(os.path.join(REF, "tests", "params_test.cpp")).read()

    def body(test):  # text of one TEST(...) block
        a = par.index(test)
        b = par.find("\nTEST(", a + 1)
        return par[a:b if b > 0 else len(par)]

    dflt = {}
    for name, val in re.findall(r"EXPECT_DOUBLE_EQ\(p\.(\w+),\s*([0-9.eE+-]+)\)",
                                body("TEST(Params, DefaultsMatchFortran)")):
        dflt[name] = float(val)
    pins["params_defaults"] = dflt
    der = {}
    for name, val in re.findall(r"EXPECT_DOUBLE_EQ\(d\.(\w+),\s*([0-9.]+)\);",
                                body("TEST(Derived, GoldenGeometry)")):
        der[name] = float(val)
    pins["derived_golden_16x16x32"] = der
    grid = open(os.path.join(REF, "tests", "grid_test.cpp")).read()
    m = re.search(r"EXPECT_NEAR\(s,\s*([0-9.]+),\s*([0-9.eE-]+)\)", grid)
    pins["mkgrid_x_1_15"] = {"value": float(m.group(1)), "tol": float(m.group(2))}

    from oracle import Reference

    runs = {}
    for name, flags, seed, nranks, steps in RUNS:
        f, _, sc, _ = Reference.run(flags, nranks=nranks, seed=seed, nsteps=steps, omp_threads=4)
        runs[name] = {"flags": flags, "seed": seed,
                      "nranks": nranks, "steps": steps,
                      "sha256_interior": {k: interior_sha(f[k]) for k in ("ru", "rv", "rw", "ro", "tt")},
                      "scalars_hex": {k: float(sc[k]).hex() for k in ("dt", "timc", "timt", "umach", "tb")},
                      "nit": int(sc["nit"])}
    pins["reference_runs"] = runs
    out = os.path.join(HERE, "reference_pins.json")
    with open(out, "w") as fh:
        json.dump(pins, fh, indent=1, sort_keys=True)
    print("wrote", out)


if __name__ == "__main__":
    main()
