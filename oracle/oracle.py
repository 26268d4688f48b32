"""ctypes front end for the two CPU checkers (test infrastructure only).

* ``Oracle``    - the C restatement in r3d_oracle.c (always available once built).
* ``Reference`` - the reference's own CPU sources compiled unmodified into
  _ref/libr3dref.so (present where the reference tree was available at build time); with
  ``run_gpu`` / ``time_gpu`` the same set-up followed by the reference's own GPU driver
  (src/gpu.cpp, src/gpu_kernels.cu for sm_100a, one copy per thread-rank, _ref/libr3dgpu_r*.so).

Both take reference-style CLI flags (src/params.cpp:113-224) and return global
(npx+2) x (npy+2) x (npz+2) arrays shaped (NZ, NY, NX).  Only tests/, the smoke check and
bench.py's CPU legs import this module.
"""
from __future__ import annotations

import ctypes
import os
from typing import Dict, List, Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libr3dref.so")
REF_GPU_COPIES = [os.path.join(HERE, "_ref", f"libr3dgpu_r{r}.so") for r in range(8)]

FIELDS = ["ru", "rv", "rw", "ro", "tt", "uu", "vv", "ww", "fu", "fv", "fw", "fr", "ft",
          "zru", "zrv", "zrw", "zro", "ztt", "ww1", "ww2", "ww3", "bx", "by", "bz",
          "zbx", "zby", "zbz"]
LINES = ["exx", "dxxdx", "d2xxdx2", "ddx", "wyy", "dyydy", "d2yydy2", "ddy",
         "zee", "dzzdz", "d2zzdz2", "ddz", "rkapa", "dkapa"]
SCALARS = ["dt", "timc", "timt", "timi", "umach", "tb", "nit"]
PRIMARY = ["ru", "rv", "rw", "ro", "tt", "bx", "by", "bz"]


def _argv(args: Sequence[str]):
    arr = (ctypes.c_char_p * len(args))(*[a.encode() for a in args])
    return arr, len(args)


def grid_of(args: Sequence[str]):
    d = {"--npx": 504, "--npy": 504, "--npz": 2048}
    a = list(args)
    for i, x in enumerate(a):
        for k in d:
            if x == k:
                d[k] = int(a[i + 1])
            elif x.startswith(k + "="):
                d[k] = int(x.split("=", 1)[1])
    return d["--npx"], d["--npy"], d["--npz"]


class Oracle:
    """The C restatement on one global domain."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            if not os.path.exists(ORACLE_SO):
                raise RuntimeError(f"oracle library missing: {ORACLE_SO} (run build())")
            lib = ctypes.CDLL(ORACLE_SO)
            lib.ora_create.restype = ctypes.c_void_p
            lib.ora_create.argtypes = [ctypes.c_int, ctypes.c_void_p]
            lib.ora_destroy.argtypes = [ctypes.c_void_p]
            lib.ora_error.restype = ctypes.c_char_p
            lib.ora_init.argtypes = [ctypes.c_void_p, ctypes.c_int]
            lib.ora_step.argtypes = [ctypes.c_void_p, ctypes.c_int]
            lib.ora_fluxes.argtypes = [ctypes.c_void_p]
            lib.ora_heat_loss.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
            lib.ora_density_diffusion.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
            lib.ora_communicate.argtypes = [ctypes.c_void_p]
            lib.ora_field.restype = ctypes.POINTER(ctypes.c_double)
            lib.ora_field.argtypes = [ctypes.c_void_p, ctypes.c_int]
            lib.ora_line.restype = ctypes.POINTER(ctypes.c_double)
            lib.ora_line.argtypes = [ctypes.c_void_p, ctypes.c_int]
            lib.ora_get_scalars.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
            lib.ora_set_scalars.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
            lib.ora_dims.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
            lib.ora_static_profile.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
            lib.ora_ran2.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
            lib.ora_mkgrid.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_void_p]
            lib.ora_param.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_void_p]
            cls._lib = lib
        return cls._lib

    def __init__(self, args: Sequence[str]):
        lib = self.lib()
        arr, n = _argv(args)
        self.h = lib.ora_create(n, arr)
        if not self.h:
            raise ValueError(lib.ora_error().decode())
        d = np.zeros(3, dtype=np.int32)
        lib.ora_dims(self.h, d.ctypes.data)
        self.NX, self.NY, self.NZ = (int(x) for x in d)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib().ora_destroy(self.h)
            self.h = None

    def _check(self, rc):
        if rc != 0:
            raise RuntimeError(self.lib().ora_error().decode())

    def init(self, seed: int = 62659):
        self._check(self.lib().ora_init(self.h, seed))
        return self

    def step(self, nstages: int = 3):
        self._check(self.lib().ora_step(self.h, nstages))

    def fluxes(self):
        self._check(self.lib().ora_fluxes(self.h))

    def communicate(self):
        self.lib().ora_communicate(self.h)

    def heat_loss(self) -> np.ndarray:
        """The itcon-2 embedded heat-loss term of the current state (FT starting from zeros),
        shape (NZ, NY, NX)."""
        out = np.zeros((self.NZ, self.NY, self.NX))
        self._check(self.lib().ora_heat_loss(self.h, out.ctypes.data))
        return out

    def density_diffusion(self) -> np.ndarray:
        """The density-diffusion terms (ID 1, 2) of the current state (FR starting from zeros),
        shape (NZ, NY, NX)."""
        out = np.zeros((self.NZ, self.NY, self.NX))
        self._check(self.lib().ora_density_diffusion(self.h, out.ctypes.data))
        return out

    def field(self, name: str) -> np.ndarray:
        """A live view of a 3D field, shape (NZ, NY, NX)."""
        ptr = self.lib().ora_field(self.h, FIELDS.index(name))
        return np.ctypeslib.as_array(ptr, shape=(self.NZ, self.NY, self.NX))

    def line(self, name: str) -> np.ndarray:
        q = LINES.index(name)
        n = self.NX if q < 4 else (self.NY if q < 8 else self.NZ)
        return np.ctypeslib.as_array(self.lib().ora_line(self.h, q), shape=(n,))

    def scalars(self) -> Dict[str, float]:
        v = np.zeros(7)
        self.lib().ora_get_scalars(self.h, v.ctypes.data)
        return dict(zip(SCALARS, v.tolist()))

    def set_scalars(self, sc: Dict[str, float]):
        v = np.array([sc[k] for k in SCALARS], dtype=np.float64)
        self.lib().ora_set_scalars(self.h, v.ctypes.data)

    def param(self, name: str) -> float:
        out = ctypes.c_double()
        if self.lib().ora_param(self.h, name.encode(), ctypes.byref(out)) != 0:
            raise KeyError(name)
        return out.value

    def static_profile(self, npz: Optional[int] = None):
        t = np.zeros(self.NZ - 2)
        r = np.zeros(self.NZ - 2)
        self._check(self.lib().ora_static_profile(self.h, t.ctypes.data, r.ctypes.data))
        return t, r

    def mkgrid(self, scode: float, icoord: int):
        o = np.zeros(3)
        self.lib().ora_mkgrid(self.h, scode, icoord, o.ctypes.data)
        return tuple(o.tolist())

    @classmethod
    def ran2(cls, seed: int, n: int) -> np.ndarray:
        o = np.zeros(n)
        cls.lib().ora_ran2(seed, n, o.ctypes.data)
        return o


class Reference:
    """The reference CPU sources (compiled unmodified) on thread-ranks."""

    _lib = None

    @classmethod
    def available(cls) -> bool:
        return os.path.exists(REF_SO)

    @classmethod
    def gpu_available(cls) -> bool:
        return cls.available() and all(os.path.exists(c) for c in REF_GPU_COPIES)

    @classmethod
    def lib(cls):
        if cls._lib is None:
            if not os.path.exists(REF_SO):
                raise RuntimeError(f"reference build missing: {REF_SO}")
            lib = ctypes.CDLL(REF_SO)
            lib.ref_run.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
            lib.ref_last_error.restype = ctypes.c_char_p
            lib.ref_ran2.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
            lib.ref_time.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
            lib.ref_run_gpu.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
            lib.ref_time_gpu.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
            cls._lib = lib
        return cls._lib

    @classmethod
    def run(cls, args: Sequence[str], nranks: int = 2, seed: int = 62659, nsteps: int = 0,
            last_stages: int = 3, omp_threads: int = 1, fluxes_only: bool = False,
            want_lines: bool = False):
        """Run set-up + nsteps reference steps; returns (fields, lines, scalars, seconds)."""
        npx, npy, npz = grid_of(args)
        NX, NY, NZ = npx + 2, npy + 2, npz + 2
        out3 = np.zeros((8, NZ, NY, NX))
        out1 = np.zeros(4 * NX + 4 * NY + 6 * NZ) if want_lines else None
        sc = np.zeros(7)
        secs = np.zeros(1)
        arr, n = _argv(args)
        rc = cls.lib().ref_run(arr, n, nranks, seed, nsteps, last_stages, omp_threads,
                               int(fluxes_only), out3.ctypes.data,
                               out1.ctypes.data if out1 is not None else None,
                               sc.ctypes.data, secs.ctypes.data)
        if rc != 0:
            raise RuntimeError(cls.lib().ref_last_error().decode())
        names = (["fu", "fv", "fw", "fr", "ft", "ro", "uu", "vv"] if fluxes_only else PRIMARY)
        fields = dict(zip(names, out3))
        lines = None
        if out1 is not None:
            lines = {}
            off = 0
            for q, nm in enumerate(LINES):
                n1 = NX if q < 4 else (NY if q < 8 else NZ)
                lines[nm] = out1[off:off + n1].copy()
                off += n1
        return fields, lines, dict(zip(SCALARS, sc.tolist())), float(secs[0])

    @classmethod
    def time_steps(cls, args: Sequence[str], nranks: int, seed: int, warmup: int, nsteps: int,
                   omp_threads: int):
        """Set-up, `warmup` untimed and `nsteps` timed reference steps without gathering the
        state; returns (scalars, seconds of the timed steps)."""
        sc = np.zeros(7)
        secs = np.zeros(1)
        arr, n = _argv(args)
        rc = cls.lib().ref_time(arr, n, nranks, seed, warmup, nsteps, omp_threads, sc.ctypes.data,
                                secs.ctypes.data)
        if rc != 0:
            raise RuntimeError(cls.lib().ref_last_error().decode())
        return dict(zip(SCALARS, sc.tolist())), float(secs[0])

    @classmethod
    def run_gpu(cls, args: Sequence[str], nranks: int = 2, seed: int = 62659, nsteps: int = 0,
                last_stages: int = 3):
        """Set-up + nsteps steps of the reference GPU driver (needs a GPU: the driver exits the
        process on a CUDA error, src/gpu.cpp:117-126); returns (fields, scalars, seconds)."""
        npx, npy, npz = grid_of(args)
        out3 = np.zeros((8, npz + 2, npy + 2, npx + 2))
        sc = np.zeros(7)
        secs = np.zeros(1)
        arr, n = _argv(args)
        rc = cls.lib().ref_run_gpu(arr, n, nranks, seed, nsteps, last_stages, out3.ctypes.data,
                                   sc.ctypes.data, secs.ctypes.data)
        if rc != 0:
            raise RuntimeError(cls.lib().ref_last_error().decode())
        return dict(zip(PRIMARY, out3)), dict(zip(SCALARS, sc.tolist())), float(secs[0])

    @classmethod
    def time_gpu(cls, args: Sequence[str], nranks: int, seed: int, warmup: int, nsteps: int):
        """Set-up, `warmup` untimed and `nsteps` timed steps of the reference GPU driver, the
        device synchronised and the ranks joined on both sides; returns (scalars, seconds)."""
        sc = np.zeros(7)
        secs = np.zeros(1)
        arr, n = _argv(args)
        rc = cls.lib().ref_time_gpu(arr, n, nranks, seed, warmup, nsteps, sc.ctypes.data, secs.ctypes.data)
        if rc != 0:
            raise RuntimeError(cls.lib().ref_last_error().decode())
        return dict(zip(SCALARS, sc.tolist())), float(secs[0])

    @classmethod
    def ran2(cls, seed: int, n: int) -> np.ndarray:
        o = np.zeros(n)
        cls.lib().ref_ran2(seed, n, o.ctypes.data)
        return o


def interior(a: np.ndarray) -> np.ndarray:
    return a[1:-1, 1:-1, 1:-1]
