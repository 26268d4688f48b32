"""Build the B200 library (lib/librast3d_b200.so) and the CLI driver (bin/r3d_b200).

nvcc compiles the device code for sm_100a only, with FMA contraction off (-fmad=false): the
FP64 step must reproduce the reference CPU arithmetic bit for bit.  Host C++ is compiled with
-ffp-contract=off for the same reason (the reference builds with it, makefile:104).
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
          "-I", os.path.join(ROOT, "include"), "-I", os.path.join(PKG, "host"), "-I", os.path.join(PKG, "csrc")]
HOST_SRCS = ["host/params.cpp", "host/setup.cpp"]
# FMA contraction: off everywhere the FP64 result must equal the reference CPU build; on for
# the FP32-bulk kernels, which carry no bit-exactness contract.
FMAD_ON = {"csrc/step_fp32.cu", "csrc/bcon_fp32.cu"}
CU_SRCS = ["csrc/step_fp64.cu", "csrc/bcon.cu", "csrc/step_fp32.cu", "csrc/bcon_fp32.cu", "csrc/r3d_gpu.cu", "csrc/dt_noalloc.cu", "csrc/adjoint.cu", "csrc/halo.cu", "csrc/mesh.cu", "csrc/compare.cu"]
LIB = os.path.join(PKG, "lib", "librast3d_b200.so")
BIN = os.path.join(PKG, "bin", "r3d_b200")


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose_ptxas: bool = False, force: bool = False) -> str:
    os.makedirs(os.path.join(PKG, "lib"), exist_ok=True)
    os.makedirs(os.path.join(PKG, "bin"), exist_ok=True)
    os.makedirs(os.path.join(PKG, "_build"), exist_ok=True)
    srcs = [s for s in CU_SRCS + HOST_SRCS if os.path.exists(os.path.join(PKG, s))]
    deps = [os.path.join(PKG, s) for s in srcs]
    for d in ("csrc", "host"):
        deps += [os.path.join(PKG, d, f) for f in os.listdir(os.path.join(PKG, d))]
    deps.append(os.path.join(ROOT, "include", "r3d_gpu.h"))
    objs = []
    for s in srcs:
        src = os.path.join(PKG, s)
        obj = os.path.join(PKG, "_build", os.path.basename(s) + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + deps):
            extra = ["-Xptxas", "-v"] if (verbose_ptxas and s.endswith(".cu")) else []
            lang = ["-x", "cu"] if s.endswith(".cu") else ["-x", "c++"]
            fmad = ["-fmad=true"] if s in FMAD_ON else ["-fmad=false"]
            omp = ["-Xcompiler", "-fopenmp"] if s in HOST_SRCS else []  # host set-up loops
            _run([NVCC] + ARCH + COMMON + fmad + omp + extra + lang + ["-c", src, "-o", obj])
    if force or _stale(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-o", LIB] + objs +
             ["-cudart", "static", "-ldl", "-lgomp"])
    main = os.path.join(PKG, "host", "r3d_main.cpp")
    if os.path.exists(main) and (force or _stale(BIN, [main, LIB])):
        _run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-I", os.path.join(ROOT, "include"),
              "-I", os.path.join(PKG, "host"), main, "-o", BIN, "-L", os.path.join(PKG, "lib"),
              "-lrast3d_b200", "-Wl,-rpath,$ORIGIN/../lib"])
    return LIB


if __name__ == "__main__":
    build(verbose_ptxas="-v" in sys.argv, force="-f" in sys.argv)
