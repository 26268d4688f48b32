"""The r3d_b200 command-line driver (rast-3dmhd_b200/host/r3d_main.cpp).

It mirrors the reference main() GPU time loop (src/main.cpp:110-275): flags, start-up line,
NIT progress lines at the NSTEP0 cadence, the dt underflow stop and gstate dumps in the
reference's binary layout (src/main.cpp:42-93).  CPU tests cover argument handling; the GPU
test runs a short job and compares the dumped state with the oracle bit for bit.
"""
import os
import struct
import subprocess

import numpy as np
import pytest

from conftest import ROOT as REPO

BIN = os.path.join(REPO, "rast-3dmhd_b200", "bin", "r3d_b200")
FIELDS27 = ["ru", "rv", "rw", "ro", "tt", "uu", "vv", "ww", "fu", "fv", "fw", "fr", "ft", "zru", "zrv",
            "zrw", "zro", "ztt", "ww1", "ww2", "ww3", "bx", "by", "bz", "zbx", "zby", "zbz"]
LINES14 = ["exx", "dxxdx", "d2xxdx2", "ddx", "wyy", "dyydy", "d2yydy2", "ddy", "zee", "dzzdz",
           "d2zzdz2", "ddz", "rkapa", "dkapa"]


def read_gstate(path):
    """Reader of the gstate layout: magic, nf, n1, 13 ints, 27 doubles, nf counted 3D arrays,
    n1 counted 1D arrays, int64 -1."""
    with open(path, "rb") as f:
        b = f.read()
    magic, nf, n1 = struct.unpack_from("<iii", b, 0)
    assert magic == 1129928788 and nf == 27 and n1 == 14
    hdr = struct.unpack_from("<13i", b, 12)
    sc = struct.unpack_from("<27d", b, 12 + 52)
    off = 12 + 52 + 216
    nx, ny, nz = hdr[:3]
    arrays = {}
    for name in FIELDS27:
        (cnt,) = struct.unpack_from("<q", b, off)
        off += 8
        assert cnt == nx * ny * nz
        arrays[name] = np.frombuffer(b, dtype="<f8", count=cnt, offset=off).reshape(nz, ny, nx)
        off += 8 * cnt
    lines = {}
    for name in LINES14:
        (cnt,) = struct.unpack_from("<q", b, off)
        off += 8
        lines[name] = np.frombuffer(b, dtype="<f8", count=cnt, offset=off)
        off += 8 * cnt
    (end,) = struct.unpack_from("<q", b, off)
    assert end == -1 and off + 8 == len(b)
    return hdr, sc, arrays, lines


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
    hdr, sc, arr, lines = read_gstate(os.path.join(tmp_path, "gstate.start.000.0000"))
    assert hdr[:3] == (22, 14, 26) and hdr[6] == 0
    for n in ("ru", "rv", "rw", "ro", "tt"):
        assert np.array_equal(interior(arr[n]), interior(o.field(n))), n
    for n in LINES14:
        assert np.array_equal(lines[n], o.line(n)), n
    for s in range(5):
        o.step()
    hdr, sc, arr, _ = read_gstate(os.path.join(tmp_path, "gstate.step.000.0005"))
    osc = o.scalars()
    assert hdr[6] == 5 and sc[0] == osc["dt"] and sc[1] == osc["timc"]
    for n in ("ru", "rv", "rw", "ro", "tt"):
        assert np.array_equal(interior(arr[n]), interior(o.field(n))), n
    # --dump-mode 0: progress lines only
    r = run(flags + ["--dump-mode", "0"], tmp_path / "..")
    assert r.returncode == 0 and sum(ln.startswith("NIT ") for ln in r.stderr.splitlines()) == 3
