"""Reader of gstate dumps, the reference's binary state format (src/main.cpp:42-93), as written
by the r3d_b200 command-line driver.

Layout (little endian): int32 magic 1129928788, int32 nf = 27, int32 n1 = 14; a 13-int header
(nx, ny, nz, three zeros, nit, lmag, ixcon, iycon, izcon, itcon, ibcon); 27 doubles (dt timc
timt timi umach re repr cv ocv ore theta grav rkapst orm rm obeta omx omz sf ampt, a zero, hx h2x
hy h2y hz h2z); nf 3D arrays and n1 1D arrays, each an int64 element count followed by the
doubles; int64 -1.  3D arrays are (nz, ny, nx) with x fastest.  The r3d_b200 driver writes the
RK accumulators zru..ztt and zbx..zbz from the device (interior cells); the FLUXES temporaries
uu..ft and ww1..ww3 do not exist in the fused kernels and are written as zeros.
"""
from __future__ import annotations

import struct
from dataclasses import dataclass
from typing import Dict

import numpy as np

MAGIC = 1129928788
FIELDS = ["ru", "rv", "rw", "ro", "tt", "uu", "vv", "ww", "fu", "fv", "fw", "fr", "ft", "zru", "zrv",
          "zrw", "zro", "ztt", "ww1", "ww2", "ww3", "bx", "by", "bz", "zbx", "zby", "zbz"]
LINES = ["exx", "dxxdx", "d2xxdx2", "ddx", "wyy", "dyydy", "d2yydy2", "ddy", "zee", "dzzdz",
         "d2zzdz2", "ddz", "rkapa", "dkapa"]
HEADER = ["nx", "ny", "nz", "pad0", "pad1", "pad2", "nit", "lmag", "ixcon", "iycon", "izcon",
          "itcon", "ibcon"]
SCALARS = ["dt", "timc", "timt", "timi", "umach", "re", "repr", "cv", "ocv", "ore", "theta", "grav",
           "rkapst", "orm", "rm", "obeta", "omx", "omz", "sf", "ampt", "pad", "hx", "h2x", "hy", "h2y",
           "hz", "h2z"]


@dataclass
class GState:
    header: Dict[str, int]
    scalars: Dict[str, float]
    fields: Dict[str, np.ndarray]   # (nz, ny, nx) views into the file's bytes (read-only)
    lines: Dict[str, np.ndarray]


def read(path: str) -> GState:
    """Parse one gstate file; raises ValueError on any layout mismatch."""
    with open(path, "rb") as f:
        b = f.read()

    def need(ok: bool, what: str):
        if not ok:
            raise ValueError(f"{path}: {what}")

    need(len(b) >= 12 + 52 + 216, "truncated header")
    magic, nf, n1 = struct.unpack_from("<iii", b, 0)
    need(magic == MAGIC, f"bad magic {magic}")
    need(nf == len(FIELDS) and n1 == len(LINES), f"unexpected array counts {nf}, {n1}")
    hdr = dict(zip(HEADER, struct.unpack_from("<13i", b, 12)))
    sc = dict(zip(SCALARS, struct.unpack_from("<27d", b, 12 + 52)))
    off = 12 + 52 + 216
    nx, ny, nz = hdr["nx"], hdr["ny"], hdr["nz"]
    fields = {}
    for name in FIELDS:
        need(off + 8 <= len(b), f"truncated before {name}")
        (cnt,) = struct.unpack_from("<q", b, off)
        off += 8
        need(cnt == nx * ny * nz and off + 8 * cnt <= len(b), f"bad length of {name}")
        fields[name] = np.frombuffer(b, dtype="<f8", count=cnt, offset=off).reshape(nz, ny, nx)
        off += 8 * cnt
    lines = {}
    for name in LINES:
        need(off + 8 <= len(b), f"truncated before {name}")
        (cnt,) = struct.unpack_from("<q", b, off)
        off += 8
        need(0 <= cnt and off + 8 * cnt <= len(b), f"bad length of {name}")
        lines[name] = np.frombuffer(b, dtype="<f8", count=cnt, offset=off)
        off += 8 * cnt
    need(off + 8 == len(b) and struct.unpack_from("<q", b, off)[0] == -1, "missing end marker")
    return GState(hdr, sc, fields, lines)
