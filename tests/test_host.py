"""Host side of the product without a GPU: the C ABI loads and exports what include/r3d_gpu.h
declares; the CLI parser equals the reference flag set; the host set-up (metrics, static IC,
seeded perturbation, ghosts) equals the oracle bit for bit; unsupported configurations and
misuse return status codes instead of exiting."""
import ctypes
import os
import random
import re

import numpy as np
import pytest

import r3d_b200 as R
from oracle import Oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "r3d_gpu.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(r3d_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = R.lib()
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), f"{n} declared in include/r3d_gpu.h but not exported"
    assert R.version().startswith("rast3d-b200")


INT_FLAGS = ["npx", "npy", "npz", "npey", "ngrid", "id", "ncol", "nrow", "ixcon", "iycon", "izcon",
             "itcon", "ibcon", "ncase", "ncasep", "ntotal", "nstep0", "nstart", "ntube"]
DBL_FLAGS = ["re", "pr", "theta", "grav", "ang", "rm", "beta", "pzp", "sigma", "polys", "tp", "tc", "xp",
             "yp", "zp", "xmax", "ymax", "zmax", "ampt", "ampb", "bfh", "bzp", "qfh", "gamma", "hh", "dh",
             "dv", "tstart", "toff", "rlax", "xx1", "xx2", "yy1", "yy2", "zz1", "zz2", "xa", "xb", "xc",
             "xd", "ya", "yb", "yc", "yd", "za", "zb", "zc", "zd", "xcent", "zcent", "rmax", "cmt",
             "lambda", "vz0"]
RENAMED = {"ry": "r_y", "a": "a_tube", "sff": "sf", "gpu": "gpu_id"}


def test_parser_matches_oracle_on_every_flag():
    rng = random.Random(7)
    args = []
    for f in INT_FLAGS:
        args += [f"--{f}", str(rng.randint(1, 9))] if rng.random() < 0.5 else [f"--{f}={rng.randint(1, 9)}"]
    for f in DBL_FLAGS + ["ry", "a", "sff"]:
        v = f"{rng.uniform(-3, 3):.6g}"
        args += [f"--{f}", v] if rng.random() < 0.5 else [f"--{f}={v}"]
    for f in ("lrot", "lmag", "lpot", "lrem", "lshr"):
        args += [f"--{f}", rng.choice(["1", "true", "yes", "on", "0", "no", "false"])]
    args += ["--backend", "gpu", "--gpu", "3"]
    p = R.parse(args)
    o = Oracle(args + [])
    for f in INT_FLAGS + DBL_FLAGS + ["ry", "a", "sff", "lrot", "lmag", "lpot", "lrem", "lshr", "gpu"]:
        attr = RENAMED.get(f, f)
        assert float(getattr(p, attr)) == o.param("--" + f), f
    assert p.backend == 1


def test_parser_rejects_unknown_and_missing_values():
    with pytest.raises(R.R3dError) as e:
        R.parse(["--bogus", "1"])
    assert e.value.code == R.R3D_EINVAL and "unknown option" in str(e.value)
    with pytest.raises(R.R3dError):
        R.parse(["--npx"])
    with pytest.raises(R.R3dError):
        R.parse(["--backend", "tpu"])
    p = R.parse(["--seed", "11", "--precision", "fp32bulk"])
    assert p.seed == 11 and p.precision == R.PREC_FP32BULK


@pytest.mark.parametrize("args,msg", [
    (["--ix", "4"], "stencil"), (["--lrem", "1"], "LREM"), (["--lshr", "1"], "LSHR"),
    (["--rlax", "0.5"], "RLAX"), (["--id", "1"], "ID"), (["--itcon", "2", "--precision", "fp32bulk"], "ITCON 2"),
    (["--itcon", "3", "--precision", "fp32bulk"], "ITCON 3"), (["--itcon", "3", "--lmag", "1"], "ITCON 3"),
    (["--itcon", "5"], "ITCON"), (["--izcon", "2"], "IZCON"),
    (["--id", "1", "--ngrid", "2"], "uniform grid"), (["--id", "3", "--ngrid", "0"], "ID must be"),
    (["--id", "1", "--ngrid", "0", "--precision", "fp32bulk"], "ID (density"),
    (["--id", "2", "--ngrid", "0", "--lmag", "1", "--beta", "10", "--rm", "1"], "ID (density"), (["--ixcon", "1"], "periodic"),
    (["--nstart", "3"], "restart"), (["--ampb", "0.1"], "AMPB"),
    (["--lmag", "1", "--rm", "0", "--beta", "1"], "LMAG"), (["--seed", "0"], "seed"),
    (["--npz", "4"], "too small"),
])
def test_unsupported_configurations_are_errors(args, msg):
    """Configurations the library refuses, with the reason (ITCON 2 and 3 run in the fp64 form)."""
    with pytest.raises(R.R3dError) as e:
        R.check(R.parse(args))
    assert e.value.code == R.R3D_EINVAL and msg in str(e.value)


SETUPS = [
    (["--npx", "32", "--npy", "32", "--npz", "64"], 1),
    (["--npx", "24", "--npy", "20", "--npz", "36", "--ngrid", "2"], 7),
    (["--npx", "24", "--npy", "20", "--npz", "36", "--ngrid", "0", "--pzp", "0.5", "--sigma", "0.1",
      "--polys", "1.5"], 3),
    (["--npx", "20", "--npy", "16", "--npz", "32", "--lmag", "1", "--beta", "10", "--rm", "1",
      "--ampb", "0.1", "--bfh", "2", "--bzp", "20"], 7),
    (["--npx", "7", "--npy", "5", "--npz", "9", "--ampt", "0"], 2),
]


@pytest.mark.parametrize("flags,seed", SETUPS)
def test_host_setup_equals_oracle_bitwise(flags, seed):
    p = R.parse(flags + ["--seed", str(seed)])
    st = R.HostState.setup(p)
    o = Oracle(flags).init(seed)
    for n, a in st.fields.items():
        assert np.array_equal(a, o.field(n)), n
    for n in R.LINES:
        assert np.array_equal(st.lines[n], o.line(n)), n
    assert st.scalars["tb"] == o.scalars()["tb"]


def test_gpu_calls_without_handle_or_upload_fail_cleanly():
    L = R.lib()
    sc = R.Scalars()
    assert L.r3d_gpu_step(None, 3, ctypes.byref(sc)) == R.R3D_EINVAL
    assert L.r3d_gpu_run(None, 1, ctypes.byref(sc)) == R.R3D_EINVAL
    assert L.r3d_gpu_destroy(None) == R.R3D_OK
    assert L.r3d_params_check(None) == R.R3D_EINVAL
