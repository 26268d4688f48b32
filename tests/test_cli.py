"""The r3d_b200 command-line driver (rast-3dmhd_b200/host/r3d_main.cpp).

It mirrors the reference main() GPU time loop (src/main.cpp:110-275): flags, start-up line,
NIT progress lines at the NSTEP0 cadence, the dt underflow stop and gstate dumps in the
reference's binary layout (src/main.cpp:42-93).  CPU tests cover argument handling; the GPU
test runs a short job and compares the dumped state with the oracle bit for bit.
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT as REPO
from r3d_b200 import gstate

BIN = os.path.join(REPO, "rast-3dmhd_b200", "bin", "r3d_b200")
def run(args, cwd, timeout=300):
    return subprocess.run([BIN] + args, cwd=cwd, capture_output=True, text=True, timeout=timeout)


def test_cli_built():
    assert os.access(BIN, os.X_OK), "build() must produce the r3d_b200 driver"


def test_cli_refuses_cpu_backend(tmp_path):
    r = run(["--npx", "8", "--npy", "8", "--npz", "8", "--backend", "cpu"], tmp_path)
    assert r.returncode != 0 and "GPU time loop only" in r.stderr


def test_cli_rejects_unknown_flag_and_bad_dump_mode(tmp_path):
    r = run(["--npx", "8", "--bogus", "1"], tmp_path)
    assert r.returncode != 0 and "argument parsing" in r.stderr
    r = run(["--npx", "8", "--dump-mode", "7"], tmp_path)
    assert r.returncode != 0 and "dump-mode" in r.stderr


def test_cli_rejects_unsupported_parameters(tmp_path):
    r = run(["--npx", "8", "--npy", "8", "--npz", "8", "--ix", "4"], tmp_path)
    assert r.returncode != 0 and "parameter check" in r.stderr


@pytest.mark.gpu
def test_cli_run_dumps_match_oracle(tmp_path):
    from oracle import Oracle, interior

    flags = ["--npx", "20", "--npy", "12", "--npz", "24", "--ntotal", "5", "--nstep0", "2"]
    r = run(flags + ["--backend", "gpu"], tmp_path)
    assert r.returncode == 0, r.stderr
    log = r.stderr.splitlines()
    assert log[0].startswith("rast-3dmhd: NP=1 NPEY=1 NPEZ=1  local 22x14x26  NIT0=5 DT=")
    nits = [int(ln.split()[1]) for ln in log if ln.startswith("NIT ")]
    assert nits == [2, 4, 5]
    names = sorted(os.listdir(tmp_path))
    assert names == ["gstate.start.000.0000", "gstate.step.000.0002", "gstate.step.000.0004",
                     "gstate.step.000.0005"]
    o = Oracle(flags).init(62659)
    g0 = gstate.read(os.path.join(tmp_path, "gstate.start.000.0000"))
    assert (g0.header["nx"], g0.header["ny"], g0.header["nz"]) == (22, 14, 26) and g0.header["nit"] == 0
    for n in ("ru", "rv", "rw", "ro", "tt"):
        assert np.array_equal(interior(g0.fields[n]), interior(o.field(n))), n
    for n in gstate.LINES:
        assert np.array_equal(g0.lines[n], o.line(n)), n
    for s in range(5):
        o.step()
    g5 = gstate.read(os.path.join(tmp_path, "gstate.step.000.0005"))
    osc = o.scalars()
    assert g5.header["nit"] == 5 and g5.scalars["dt"] == osc["dt"] and g5.scalars["timc"] == osc["timc"]
    for n in ("ru", "rv", "rw", "ro", "tt"):
        assert np.array_equal(interior(g5.fields[n]), interior(o.field(n))), n
    # the RK accumulators, on the planes strictly inside (the top and bottom planes' momentum
    # and energy accumulators follow fluxes that BCON overwrites, which the fused kernel skips)
    strict = (slice(2, -2), slice(1, -1), slice(1, -1))
    for n in ("zru", "zrv", "zrw", "zro", "ztt"):
        assert np.array_equal(g5.fields[n][strict], o.field(n)[strict]), n
    assert np.abs(g5.fields["zro"][strict]).max() > 0
    # the FLUXES work arrays of the fifth step's third stage: the velocities on every cell, the
    # right-hand sides on the interior (momentum and energy on the planes strictly inside; the
    # fused kernel leaves them 0 on the top and bottom planes, which BCON overrides)
    for n in ("uu", "vv", "ww"):
        assert np.array_equal(g5.fields[n], o.field(n)), n
    assert np.array_equal(interior(g5.fields["fr"]), interior(o.field("fr")))
    for n in ("fu", "fv", "fw", "ft"):
        assert np.array_equal(g5.fields[n][strict], o.field(n)[strict]), n
        assert not g5.fields[n][1].any() and not g5.fields[n][-2].any(), n
    assert np.abs(g5.fields["ft"][strict]).max() > 0 and np.abs(g5.fields["uu"]).max() > 0
    for n in ("ww1", "ww2", "ww3"):
        assert not g5.fields[n].any(), n
    # --dump-mode 0: progress lines only
    r = run(flags + ["--dump-mode", "0"], tmp_path / "..")
    assert r.returncode == 0 and sum(ln.startswith("NIT ") for ln in r.stderr.splitlines()) == 3


def test_gstate_reader_rejects_damaged_files(tmp_path):
    """The reader checks magic, counts, array lengths and the end marker."""
    import struct
    nx, ny, nz = 3, 2, 2
    parts = [struct.pack("<iii", gstate.MAGIC, 27, 14), struct.pack("<13i", nx, ny, nz, *([0] * 10)),
             struct.pack("<27d", *([0.5] * 27))]
    for _ in range(27):
        parts += [struct.pack("<q", nx * ny * nz), np.arange(nx * ny * nz, dtype="<f8").tobytes()]
    for _ in range(14):
        parts += [struct.pack("<q", 4), np.ones(4, dtype="<f8").tobytes()]
    good = b"".join(parts + [struct.pack("<q", -1)])
    (tmp_path / "ok").write_bytes(good)
    g = gstate.read(str(tmp_path / "ok"))
    assert g.fields["ro"].shape == (nz, ny, nx) and g.fields["tt"][1, 1, 2] == 11.0
    assert g.scalars["dt"] == 0.5 and list(g.lines) == gstate.LINES
    for bad in (good[:-8], b"\0" * 4 + good[4:], good[:200]):
        (tmp_path / "bad").write_bytes(bad)
        with pytest.raises(ValueError):
            gstate.read(str(tmp_path / "bad"))


def test_cli_restart_refuses_missing_or_mismatched_dumps(tmp_path):
    """--nstart k reads the dump written at NIT = k * nstep0 (the Fortran driver's dump index,
    3dmhd.f:289-365); a missing file or another grid is refused before any GPU work."""
    r = run(["--npx", "8", "--npy", "8", "--npz", "8", "--nstart", "2", "--nstep0", "5"], tmp_path)
    assert r.returncode != 0 and "gstate.step.000.0010" in r.stderr and "not found" in r.stderr
    import struct
    nx, ny, nz = 5, 5, 5  # a dump of another grid
    parts = [struct.pack("<iii", gstate.MAGIC, 27, 14), struct.pack("<13i", nx, ny, nz, *([0] * 10)),
             struct.pack("<27d", *([0.5] * 27))]
    (tmp_path / "gstate.step.000.0010").write_bytes(b"".join(parts))
    r = run(["--npx", "8", "--npy", "8", "--npz", "8", "--nstart", "2", "--nstep0", "5"], tmp_path)
    assert r.returncode != 0 and "grid size mismatch" in r.stderr


@pytest.mark.gpu
def test_cli_restart_continues_the_run_bit_for_bit(tmp_path):
    """A run restarted from its NIT-5 dump reaches the continuous run's NIT-10 state bit for bit
    (the dumps hold whole arrays, ghost planes included); time restarts from TIMI = TIMI + TIMC
    of the dump with TIMC = 0, as in the Fortran driver."""
    from oracle import interior

    flags = ["--npx", "20", "--npy", "12", "--npz", "24", "--nstep0", "5"]
    a, b = tmp_path / "continuous", tmp_path / "restarted"
    a.mkdir()
    b.mkdir()
    r = run(flags + ["--ntotal", "10"], a)
    assert r.returncode == 0, r.stderr
    r = run(flags + ["--ntotal", "5"], b)
    assert r.returncode == 0, r.stderr
    r = run(flags + ["--ntotal", "5", "--nstart", "1"], b)
    assert r.returncode == 0, r.stderr
    assert [ln.split()[1] for ln in r.stderr.splitlines() if ln.startswith("NIT ")] == ["10"]
    ga = gstate.read(str(a / "gstate.step.000.0010"))
    gb = gstate.read(str(b / "gstate.step.000.0010"))
    assert ga.header == gb.header and ga.header["nit"] == 10
    for n in ("ru", "rv", "rw", "ro", "tt"):  # whole arrays, ghosts included
        assert np.array_equal(ga.fields[n], gb.fields[n]), n
    for n in ("zru", "zrv", "zrw", "zro", "ztt"):  # the accumulators are kept on interior cells
        assert np.array_equal(interior(ga.fields[n]), interior(gb.fields[n])), n
    assert ga.scalars["dt"] == gb.scalars["dt"]
    g5 = gstate.read(str(b / "gstate.step.000.0005"))
    assert gb.scalars["timi"] == g5.scalars["timi"] + g5.scalars["timc"]
    assert abs(gb.scalars["timi"] + gb.scalars["timc"] - ga.scalars["timc"]) <= 1e-14 * ga.scalars["timc"]
