"""Fixture of the density diffusion (ID 1 and 2): the reference's Fortran block executed statement
by statement (test infrastructure).

Density diffusion exists only in the Fortran FLUXES (golden/fortran/3dmhdsub.f:1316-1386); the
reference C++ aborts on --id (src/fluxes.cpp:46-51).  For each case below, on the oracle's state
after a few steps (rho in RO, as at the start of FLUXES):

* the two ghost-plane mirror statements (3dmhdsub.f:1318, 1321, array sections) and the
  uniform-grid HORIZONTAL_MEAN (3dmhdsub.f:3177-3186, with a single rank in y) are checked
  against their source text and carried out here as written (sequential sums in loop order);
* the loop `DO 9120` (WW1 = RO - ROM, 3dmhdsub.f:1326-1330) and the whole `IF (ID.NE.0)` block
  (3dmhdsub.f:1332-1386) are executed from the source text by oracle/fortran_lmag.py;

the resulting FR (from zeros) is stored in tests/golden/id_diffusion_golden.npz.

    python tests/golden/make_id_golden.py <reference checkout>     (or set R3D_REFERENCE)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import fortran_lmag  # noqa: E402
from fortran_lmag import Block, read_block  # noqa: E402
from oracle import Oracle  # noqa: E402

# the reference checkout: the first argument when run as a script, else $R3D_REFERENCE (no default)
REF = sys.argv[1] if len(sys.argv) > 1 and __name__ == "__main__" else os.environ.get("R3D_REFERENCE", "")
BASE = ["--ngrid", "0"]
CASES = {
    # name: (flags, seed, steps before the evaluation); DH, DV exact in single precision
    "id1_dh_12x10x16_seed3_2steps": (["--npx", "12", "--npy", "10", "--npz", "16", "--id", "1",
                                      "--dh", "0.5"] + BASE, 3, 2),
    "id1_dv_9x11x13_seed5_3steps": (["--npx", "9", "--npy", "11", "--npz", "13", "--id", "1",
                                     "--dv", "0.75"] + BASE, 5, 3),
    "id2_dh_dv_10x8x20_seed7_2steps": (["--npx", "10", "--npy", "8", "--npz", "20", "--id", "2",
                                        "--dh", "0.25", "--dv", "0.25", "--zmax", "1"] + BASE, 7, 2),
}
# the statements carried out in Python, as they read in the source
MIRROR = {1318: "RO(:,:,1:ILAP/2)=RO(:,:,ILAP/2+2:ILAP+1)", 1321: "RO(:,:,NZ-ILAP/2+1:NZ)=RO(:,:,NZ-ILAP:NZ-ILAP/2-1)"}
MEAN = [("", "IF(NGRID.EQ.0) THEN"), ("", "DO K=1,NZ"), ("", "WWZ(K)=0.0"), ("", "DO J=IY/2+1,NY-IY/2"),
        ("", "DO I=IX/2+1,NX-IX/2"), ("", "WWZ(K)=WWZ(K)+VAR(I,J,K)"), ("", "END DO"), ("", "END DO"),
        ("", "WWZ(K)=WWZ(K)/(FLOAT(NPX*NPY))"), ("", "END DO")]


def source(path):
    """Check the statements done in Python against the source and return the two executable
    blocks: the loop DO 9120 and the IF (ID.NE.0) block."""
    for line, text in MIRROR.items():
        got = read_block(path, line, line)
        assert [s for _, s in got] == [text], (line, got)
    got = [(lab, s.replace(" ", "")) for lab, s in read_block(path, 3177, 3186)]
    assert got == [(lab, s.replace(" ", "")) for lab, s in MEAN], got
    assert [s for _, s in read_block(path, 1324, 1324)] == ["CALL HORIZONTAL_MEAN(ROM,RO)"]
    ww1 = Block.__new__(Block)
    ww1.stmts = [("", "IF (ID.NE.0) THEN")] + read_block(path, 1326, 1330) + [("", "ENDIF")]
    return ww1, Block(path, 1332, 1386, guard="ID.NE.0")


def horizontal_mean(var, npx, npy):
    """HORIZONTAL_MEAN, NGRID = 0, one rank in y (3dmhdsub.f:3177-3186, 3211-3212), as written."""
    nz, ny, nx = var.shape
    out = np.zeros(nz)
    cnt = float(np.float32(npx * npy))  # FLOAT(NPX*NPY)
    for k in range(nz):
        s = 0.0
        for j in range(1, ny - 1):
            for i in range(1, nx - 1):
                s = s + float(var[k, j, i])
        out[k] = s / cnt
    return out


def fortran_diffusion(blocks, flags, seed, steps):
    ww1_block, id_block = blocks
    o = Oracle(flags).init(seed)
    for _ in range(steps):
        o.step()
    get = dict(zip(flags[::2], flags[1::2]))
    ro = o.field("ro").copy()
    ro[0] = ro[2]      # 1318, MYPEZ = 0 (ILAP = 2)
    ro[-1] = ro[-3]    # 1321, MYPEZ = NPEZ - 1
    env = {"RO": ro, "ROM": horizontal_mean(ro, int(get["--npx"]), int(get["--npy"])),
           "WW1": np.zeros_like(ro), "WW2": np.zeros_like(ro), "WW3": np.zeros_like(ro), "FR": np.zeros_like(ro)}
    for n in ("dxxdx", "d2xxdx2", "dyydy", "d2yydy2", "dzzdz", "d2zzdz2", "zee"):
        env[n.upper()] = np.array(o.line(n))
    for k in ("hx", "h2x", "hy", "h2y", "hz", "h2z", "ore"):
        env[k.upper()] = o.param(k)
    env.update(ID=int(get["--id"]), DH=float(get.get("--dh", 0.0)), DV=float(get.get("--dv", 0.0)),
               ZMAX=o.param("--zmax"), ILAP=2, IX=2, IY=2, NX=o.NX, NY=o.NY, NZ=o.NZ, MYPEZ=0, NPEZ=2)
    ww1_block.run(env)
    id_block.run(env)
    return o, env["FR"]


def main():
    if not REF or not os.path.isdir(os.path.join(REF, "golden")):
        sys.exit("usage: make_id_golden.py <reference checkout> (or set R3D_REFERENCE)")
    blocks = source(os.path.join(REF, "golden", "fortran", "3dmhdsub.f"))
    data = {}
    for name, (flags, seed, steps) in CASES.items():
        _, fr = fortran_diffusion(blocks, flags, seed, steps)
        data[name] = fr[1:-1, 1:-1, 1:-1]
    np.savez_compressed(os.path.join(HERE, "id_diffusion_golden.npz"), **data)
    print("wrote", len(data), "arrays")


if __name__ == "__main__":
    main()
