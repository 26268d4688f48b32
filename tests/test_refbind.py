"""The reference's own driver with the B200 library behind `--backend gpu`.

oracle/_ref/r3d_ref_gpu is the reference's src/main.cpp, compiled unmodified together with its
CPU sources and rast-3dmhd_b200/refbind/gpu_shim.cpp (the reference's gpu_alloc / gpu_upload /
step_gpu / gpu_download / gpu_free, include/gpu.hpp:35-49, over the C ABI), run on thread-ranks
of the MPI stand-in (oracle/Makefile target refgpu).  One binary runs both backends, so the
gstate dumps of `--backend gpu` and `--backend cpu` of one job must agree bit for bit, as the
reference's own tests/gpu_equivalence_test.cpp:143-174 requires of its CUDA path: the state
interiors (x/y ghost images included), the scalars and the header, and the RK accumulators
zru..ztt on the planes strictly inside the domain (on the top and bottom planes the reference
keeps momentum and energy fluxes that BCON overwrites; the fused kernel does not form them, so
only the accumulator values there - never the state - differ), and the FLUXES work arrays of
the last third stage: uu vv ww on every cell, FR on each rank's interior and FU FV FW FT on its
planes strictly inside.
"""
import glob
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from r3d_b200 import gstate

BIN = os.path.join(ROOT, "oracle", "_ref", "r3d_ref_gpu")
PRIMARY = ["ru", "rv", "rw", "ro", "tt"]
ACCUM = ["zru", "zrv", "zrw", "zro", "ztt"]

needs_bin = pytest.mark.skipif(not os.access(BIN, os.X_OK), reason="reference driver binding not built")


def run(backend, nranks, flags, cwd, env_extra=None, timeout=600):
    env = dict(os.environ, R3D_NRANKS=str(nranks), OMP_NUM_THREADS="2")
    env.update(env_extra or {})
    r = subprocess.run([BIN] + flags + ["--backend", backend], cwd=cwd, capture_output=True, text=True,
                       timeout=timeout, env=env)
    return r


@needs_bin
def test_cpu_backend_runs_the_reference_loop(tmp_path):
    """The CPU branch of the same binary: the reference's own time loop and dumps."""
    r = run("cpu", 2, ["--npx", "16", "--npy", "16", "--npz", "32", "--npey", "1", "--ntotal", "4",
                       "--nstep0", "2"], tmp_path)
    assert r.returncode == 0, r.stderr
    assert "NP=2 NPEY=1 NPEZ=2" in r.stderr and "NIT 4" in r.stderr
    assert sorted(os.path.basename(f) for f in glob.glob(str(tmp_path / "gstate.step.*"))) == [
        "gstate.step.000.0002", "gstate.step.000.0004", "gstate.step.001.0002", "gstate.step.001.0004"]


CASES = [
    # (name, flags, ranks): config 1 on the decomposition the reference runs it on (npey 1,
    # npez 2); a 2 x 2 rank grid (y and z both split); a ragged grid with a flux bottom
    ("config1_32x32x64_npez2", ["--npx", "32", "--npy", "32", "--npz", "64", "--npey", "1", "--ntotal", "20",
                                "--nstep0", "10"], 2),
    ("grid16_2x2_ranks", ["--npx", "16", "--npy", "16", "--npz", "32", "--npey", "2", "--ntotal", "6",
                          "--nstep0", "3"], 4),
    ("ragged_izcon1", ["--npx", "21", "--npy", "12", "--npz", "24", "--npey", "1", "--izcon", "1", "--ntotal", "5",
                       "--nstep0", "5"], 3),
]


@pytest.mark.gpu
@needs_bin
@pytest.mark.parametrize("name,flags,ranks", CASES, ids=[c[0] for c in CASES])
def test_gpu_backend_dumps_equal_cpu_backend(name, flags, ranks, tmp_path):
    dirs = {}
    for backend in ("cpu", "gpu"):
        d = tmp_path / backend
        d.mkdir()
        r = run(backend, ranks, flags, d)
        assert r.returncode == 0, f"{backend}: {r.stderr[-2000:]}"
        dirs[backend] = d
        log = [ln for ln in r.stderr.splitlines() if ln.startswith("NIT ")]
        assert log, r.stderr
        dirs[backend + "_log"] = log
    # the progress lines (dt, timc, umach at 6 digits) agree
    assert [ln.split("WALL")[0] for ln in dirs["cpu_log"]] == [ln.split("WALL")[0] for ln in dirs["gpu_log"]]
    files = sorted(os.path.basename(f) for f in glob.glob(str(dirs["cpu"] / "gstate.*")))
    assert files == sorted(os.path.basename(f) for f in glob.glob(str(dirs["gpu"] / "gstate.*")))
    assert any(".step." in f for f in files)
    inner = (slice(1, -1), slice(None), slice(None))           # every plane but the z ghosts
    strict = (slice(2, -2), slice(1, -1), slice(1, -1))        # planes strictly inside
    for f in files:
        c, g = gstate.read(str(dirs["cpu"] / f)), gstate.read(str(dirs["gpu"] / f))
        assert c.header == g.header, f
        for k in ("dt", "timc", "timt", "umach"):
            assert c.scalars[k] == g.scalars[k], (f, k, c.scalars[k], g.scalars[k])
        for n in PRIMARY:
            a, b = c.fields[n][inner], g.fields[n][inner]
            assert np.array_equal(a, b), f"{f} {n}: max |gpu - cpu| = {float(np.abs(a - b).max()):.3e}"
        if ".step." in f:
            for n in ACCUM:
                a, b = c.fields[n][strict], g.fields[n][strict]
                assert np.array_equal(a, b), f"{f} {n}: max |gpu - cpu| = {float(np.abs(a - b).max()):.3e}"
                assert np.abs(a).max() > 0.0 or n == "zrw", (f, n)
            # the FLUXES work arrays of the last third stage: velocities on every cell, the
            # right-hand sides on each rank's interior (momentum and energy strictly inside)
            for n in ("uu", "vv", "ww"):
                a, b = c.fields[n], g.fields[n]
                assert np.array_equal(a, b), f"{f} {n}: max |gpu - cpu| = {float(np.abs(a - b).max()):.3e}"
            interior3 = (slice(1, -1), slice(1, -1), slice(1, -1))
            for n, sl in (("fr", interior3), ("fu", strict), ("fv", strict), ("fw", strict), ("ft", strict)):
                a, b = c.fields[n][sl], g.fields[n][sl]
                assert np.array_equal(a, b), f"{f} {n}: max |gpu - cpu| = {float(np.abs(a - b).max()):.3e}"
        for n in gstate.LINES:
            assert np.array_equal(c.lines[n], g.lines[n]), (f, n)


@pytest.mark.gpu
@needs_bin
def test_gpu_backend_fp32bulk_through_the_reference_driver(tmp_path):
    """R3D_GPU_PRECISION=fp32bulk puts the FP32-bulk form behind the same --backend gpu loop:
    the dumped state stays within the FP32-bulk error bar of the CPU run (rel L2 <= 1e-5)."""
    flags = ["--npx", "32", "--npy", "32", "--npz", "64", "--npey", "1", "--ntotal", "20", "--nstep0", "20"]
    out = {}
    for backend, extra in (("cpu", None), ("gpu", {"R3D_GPU_PRECISION": "fp32bulk"})):
        d = tmp_path / backend
        d.mkdir()
        r = run(backend, 2, flags, d, extra)
        assert r.returncode == 0, r.stderr[-2000:]
        out[backend] = d
    for rank in ("000", "001"):
        c = gstate.read(str(out["cpu"] / f"gstate.step.{rank}.0020"))
        g = gstate.read(str(out["gpu"] / f"gstate.step.{rank}.0020"))
        for n in PRIMARY:
            a, b = c.fields[n][1:-1, 1:-1, 1:-1], g.fields[n][1:-1, 1:-1, 1:-1]
            rel = float(np.linalg.norm(b - a) / np.linalg.norm(a))
            assert rel <= 1e-5, (rank, n, rel)
        assert abs(g.scalars["timc"] - c.scalars["timc"]) <= 1e-6 * c.scalars["timc"]
