"""Python binding of the B200 Rast-3DMHD step (ctypes over include/r3d_gpu.h).

This is the host-side mirror of the reference's driver interface (src/main.cpp:125-275): parse
the reference command line into a parameter struct, build the initial state on the host,
upload it, step on the GPU, download.  All compute runs in lib/librast3d_b200.so; there is no
Python or CPU fallback: if the library is missing or no CUDA device is present the calls
raise.

    p = r3d_b200.parse(["--npx", "32", "--npy", "32", "--npz", "64"])
    st = r3d_b200.HostState.setup(p)          # metrics + static IC (host, once)
    sim = r3d_b200.GpuSim(p)                   # gpu_alloc
    sim.upload(st)                             # gpu_upload
    sc = sim.step()                            # step_gpu: dt, timc, nit, ...
    sim.download(st)                           # gpu_download
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass
from typing import Dict, Optional, Sequence

import numpy as np

_PKG = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
LIB_PATH = os.path.join(_PKG, "lib", "librast3d_b200.so")

R3D_OK, R3D_EINVAL, R3D_ECUDA, R3D_ENOMEM, R3D_ESTATE, R3D_ENUMERIC = 0, -1, -2, -3, -4, -5
PREC_FP64, PREC_FP32BULK = 0, 1

_INTS1 = ["npx", "npy", "npz", "npey", "ix", "iy", "ilap", "ipad", "ngrid", "id", "ncol", "nrow",
          "ixcon", "iycon", "izcon", "itcon", "ibcon", "lrot", "lmag", "lpot", "lrem", "lshr",
          "ncase", "ncasep", "ntotal", "nstep0", "nstart", "ntube"]
_DBLS = ["re", "pr", "theta", "grav", "r_y", "ang", "rm", "beta", "pzp", "sigma", "polys", "tp",
         "tc", "xp", "yp", "zp", "xmax", "ymax", "zmax", "ampt", "ampb", "bfh", "bzp", "qfh",
         "gamma", "hh", "dh", "dv", "tstart", "toff", "rlax", "xx1", "xx2", "yy1", "yy2", "zz1",
         "zz2", "xa", "xb", "xc", "xd", "ya", "yb", "yc", "yd", "za", "zb", "zc", "zd", "xcent",
         "zcent", "rmax", "cmt", "a_tube", "lambda", "vz0", "sf"]
_INTS2 = ["backend", "gpu_id", "seed", "precision"]


class Params(ctypes.Structure):
    """r3d_params (mirrors the reference Params, include/params.hpp:24-120)."""
    _fields_ = ([(n, ctypes.c_int) for n in _INTS1] + [(n, ctypes.c_double) for n in _DBLS]
                + [(n, ctypes.c_int) for n in _INTS2])

    def as_dict(self) -> Dict[str, float]:
        return {n: getattr(self, n) for n, _ in self._fields_}


class Scalars(ctypes.Structure):
    _fields_ = [("dt", ctypes.c_double), ("timc", ctypes.c_double), ("timt", ctypes.c_double),
                ("timi", ctypes.c_double), ("umach", ctypes.c_double), ("tb", ctypes.c_double),
                ("nit", ctypes.c_int)]

    def as_dict(self) -> Dict[str, float]:
        return {n: getattr(self, n) for n, _ in self._fields_}


FIELDS3D = ["ru", "rv", "rw", "ro", "tt", "bx", "by", "bz"]
LINES = ["exx", "dxxdx", "d2xxdx2", "ddx", "wyy", "dyydy", "d2yydy2", "ddy",
         "zee", "dzzdz", "d2zzdz2", "ddz", "rkapa", "dkapa"]


class _HostStateC(ctypes.Structure):
    _fields_ = [(n, ctypes.POINTER(ctypes.c_double)) for n in FIELDS3D + LINES]


class Timing(ctypes.Structure):
    _fields_ = [("total_ms", ctypes.c_double), ("stage_ms", ctypes.c_double),
                ("bcon_ms", ctypes.c_double), ("other_ms", ctypes.c_double),
                ("stage_launches", ctypes.c_int), ("total_launches", ctypes.c_int)]


class R3dError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"r3d error {code}: {msg}")
        self.code = code


_lib = None


def lib():
    """Load librast3d_b200.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} not built; run __graft_entry__.build()")
        L = ctypes.CDLL(LIB_PATH)
        vp, ip = ctypes.c_void_p, ctypes.c_int
        L.r3d_params_default.argtypes = [ctypes.POINTER(Params)]
        L.r3d_params_parse.argtypes = [ip, ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(Params)]
        L.r3d_params_check.argtypes = [ctypes.POINTER(Params)]
        L.r3d_derived_get.argtypes = [ctypes.POINTER(Params), ctypes.c_char_p, ctypes.POINTER(ctypes.c_double)]
        L.r3d_dims.argtypes = [ctypes.POINTER(Params)] + [ctypes.POINTER(ctypes.c_int64)] * 3
        L.r3d_setup_host.argtypes = [ctypes.POINTER(Params), ctypes.POINTER(_HostStateC), ctypes.POINTER(Scalars)]
        L.r3d_static_profile.argtypes = [ctypes.POINTER(Params), vp, vp]
        L.r3d_gpu_create.argtypes = [ctypes.POINTER(Params), ctypes.POINTER(vp)]
        L.r3d_gpu_upload.argtypes = [vp, ctypes.POINTER(_HostStateC), ctypes.POINTER(Scalars)]
        L.r3d_gpu_download.argtypes = [vp, ctypes.POINTER(_HostStateC), ctypes.POINTER(Scalars)]
        L.r3d_gpu_destroy.argtypes = [vp]
        L.r3d_gpu_memory.argtypes = [vp, ctypes.POINTER(ctypes.c_int64)]
        L.r3d_gpu_plan.argtypes = [ctypes.POINTER(Params), ip, ip, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
        L.r3d_gpu_stream.argtypes = [vp]
        L.r3d_gpu_stream.restype = vp
        L.r3d_gpu_step.argtypes = [vp, ip, ctypes.POINTER(Scalars)]
        L.r3d_gpu_run.argtypes = [vp, ip, ctypes.POINTER(Scalars)]
        L.r3d_gpu_enqueue.argtypes = [vp, ip]
        L.r3d_gpu_run_timed.argtypes = [vp, ip, ctypes.POINTER(Scalars), ctypes.POINTER(Timing)]
        L.r3d_gpu_totals.argtypes = [vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
        L.r3d_gpu_compare.argtypes = [vp, vp, ctypes.c_void_p]
        L.r3d_gpu_setup.argtypes = [vp, ctypes.POINTER(Scalars)]
        L.r3d_gpu_download_accumulators.argtypes = [vp, ctypes.POINTER(ctypes.c_void_p)]
        L.r3d_gpu_debug_tma_extra.argtypes = [vp, ctypes.c_uint]
        L.r3d_gpu_debug_dt_filter.argtypes = [vp, ctypes.c_double, ctypes.POINTER(ctypes.c_int)]
        L.r3d_gpu_fluxes.argtypes = [vp, ctypes.POINTER(ctypes.POINTER(ctypes.c_double))]
        L.r3d_gpu_download_work.argtypes = [vp, ctypes.POINTER(ctypes.POINTER(ctypes.c_double))]
        L.r3d_setup_host_slab.argtypes = [ctypes.POINTER(Params), ip, ip, ctypes.POINTER(_HostStateC),
                                          ctypes.POINTER(Scalars)]
        L.r3d_gpu_create_slab.argtypes = [ctypes.POINTER(Params), ip, ip, ctypes.POINTER(vp)]
        L.r3d_nccl_unique_id.argtypes = [ctypes.c_char_p, ctypes.c_size_t]
        L.r3d_gpu_halo_init.argtypes = [vp, ctypes.c_char_p, ctypes.c_size_t, ip, ip]
        L.r3d_mesh_create.argtypes = [ctypes.POINTER(Params), ip, ctypes.POINTER(vp)]
        L.r3d_mesh_slab.argtypes = [vp, ip, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
        L.r3d_mesh_upload.argtypes = [vp, ctypes.POINTER(_HostStateC), ctypes.POINTER(Scalars)]
        L.r3d_mesh_step.argtypes = [vp, ip, ctypes.POINTER(Scalars)]
        L.r3d_mesh_run.argtypes = [vp, ip, ctypes.POINTER(Scalars)]
        L.r3d_mesh_download.argtypes = [vp, ctypes.POINTER(_HostStateC), ctypes.POINTER(Scalars)]
        L.r3d_mesh_destroy.argtypes = [vp]
        L.r3d_mesh_debug_dt_filter.argtypes = [vp, ctypes.c_double, ctypes.POINTER(ctypes.c_int)]
        dpp = ctypes.POINTER(ctypes.POINTER(ctypes.c_double))
        L.r3d_gpu_adjoint_record.argtypes = [vp, ip, ip, ctypes.POINTER(Scalars)]
        L.r3d_gpu_adjoint_backward.argtypes = [vp, dpp, dpp]
        L.r3d_gpu_adjoint_step.argtypes = [vp, dpp, dpp]
        L.r3d_gpu_adjoint_memory.argtypes = [vp, ctypes.POINTER(ctypes.c_int64)]
        L.r3d_last_error.restype = ctypes.c_char_p
        L.r3d_version.restype = ctypes.c_char_p
        _lib = L
    return _lib


def _check(rc: int):
    if rc != R3D_OK:
        raise R3dError(rc, lib().r3d_last_error().decode())


def default_params() -> Params:
    p = Params()
    _check(lib().r3d_params_default(ctypes.byref(p)))
    return p


def parse(args: Sequence[str], base: Optional[Params] = None) -> Params:
    """Reference command line (src/params.cpp:113-224) + --seed/--precision -> Params."""
    p = default_params() if base is None else base
    arr = (ctypes.c_char_p * max(1, len(args)))(*[a.encode() for a in args])
    _check(lib().r3d_params_parse(len(args), arr, ctypes.byref(p)))
    return p


def check(p: Params):
    _check(lib().r3d_params_check(ctypes.byref(p)))


def derived(p: Params, name: str) -> float:
    out = ctypes.c_double()
    _check(lib().r3d_derived_get(ctypes.byref(p), name.encode(), ctypes.byref(out)))
    return out.value


def dims(p: Params):
    n = [ctypes.c_int64() for _ in range(3)]
    _check(lib().r3d_dims(ctypes.byref(p), *[ctypes.byref(x) for x in n]))
    return tuple(int(x.value) for x in n)


def plan(p: Params, nloc: int = 0, num_sms: int = 0):
    """(z planes per CTA, tile rows) of the stage kernels for a handle over nloc planes (0: npz)
    on a device with num_sms multiprocessors (0: read from device p.gpu_id)."""
    k, r = ctypes.c_int(), ctypes.c_int()
    _check(lib().r3d_gpu_plan(ctypes.byref(p), nloc, num_sms, ctypes.byref(k), ctypes.byref(r)))
    return k.value, r.value


def static_profile(p: Params):
    t = np.zeros(p.npz)
    r = np.zeros(p.npz)
    _check(lib().r3d_static_profile(ctypes.byref(p), t.ctypes.data, r.ctypes.data))
    return t, r


@dataclass
class HostState:
    """Host arrays on the global domain, shapes (NZ, NY, NX) and (N,) for lines."""
    fields: Dict[str, np.ndarray]
    lines: Dict[str, np.ndarray]
    scalars: Dict[str, float]

    @classmethod
    def empty(cls, p: Params) -> "HostState":
        NX, NY, NZ = dims(p)
        names = FIELDS3D if p.lmag else FIELDS3D[:5]
        fields = {n: np.zeros((NZ, NY, NX)) for n in names}
        lines = {}
        for q, n in enumerate(LINES):
            lines[n] = np.zeros(NX if q < 4 else (NY if q < 8 else NZ))
        return cls(fields, lines, {})

    @classmethod
    def empty_slab(cls, p: Params, nz: int) -> "HostState":
        """Arrays for the z slab of nz planes: nz+2 planes, z lines of nz+2 entries."""
        NX, NY, _ = dims(p)
        names = FIELDS3D if p.lmag else FIELDS3D[:5]
        fields = {n: np.zeros((nz + 2, NY, NX)) for n in names}
        lines = {}
        for q, n in enumerate(LINES):
            lines[n] = np.zeros(NX if q < 4 else (NY if q < 8 else nz + 2))
        return cls(fields, lines, {})

    @classmethod
    def setup_slab(cls, p: Params, z0: int, nz: int) -> "HostState":
        """The initial state on global planes z0 .. z0+nz+1 (r3d_setup_host_slab)."""
        st = cls.empty_slab(p, nz)
        sc = Scalars()
        c = st._c()
        _check(lib().r3d_setup_host_slab(ctypes.byref(p), z0, nz, ctypes.byref(c), ctypes.byref(sc)))
        st.scalars = sc.as_dict()
        return st

    def slab_view(self, z0: int, nz: int) -> "HostState":
        """Views (no copy) of this global state on planes z0 .. z0+nz+1."""
        f = {n: a[z0:z0 + nz + 2] for n, a in self.fields.items()}
        ln = {n: (a[z0:z0 + nz + 2] if q >= 8 else a) for q, (n, a) in enumerate(
            (m, self.lines[m]) for m in LINES)}
        return HostState(f, ln, dict(self.scalars))

    @classmethod
    def setup(cls, p: Params) -> "HostState":
        """Grid metrics, conductivity, static IC, seeded perturbation, periodic ghosts."""
        st = cls.empty(p)
        sc = Scalars()
        c = st._c()
        _check(lib().r3d_setup_host(ctypes.byref(p), ctypes.byref(c), ctypes.byref(sc)))
        st.scalars = sc.as_dict()
        return st

    def _c(self) -> _HostStateC:
        c = _HostStateC()
        dp = ctypes.POINTER(ctypes.c_double)
        for n in FIELDS3D:
            a = self.fields.get(n)
            if a is not None:
                assert a.flags.c_contiguous and a.dtype == np.float64
                setattr(c, n, a.ctypes.data_as(dp))
        for n in LINES:
            a = self.lines[n]
            setattr(c, n, a.ctypes.data_as(dp))
        return c

    def copy(self) -> "HostState":
        return HostState({k: v.copy() for k, v in self.fields.items()},
                         {k: v.copy() for k, v in self.lines.items()}, dict(self.scalars))


class GpuSim:
    """Device-resident simulation (replaces GpuSim + gpu_alloc/upload/step_gpu/download/free)."""

    def __init__(self, p: Params, slab=None):
        """slab=(z0, nz): a handle over global planes z0+1 .. z0+nz (r3d_gpu_create_slab)."""
        self.p = p
        self.slab = slab
        h = ctypes.c_void_p()
        if slab is None:
            _check(lib().r3d_gpu_create(ctypes.byref(p), ctypes.byref(h)))
        else:
            _check(lib().r3d_gpu_create_slab(ctypes.byref(p), int(slab[0]), int(slab[1]), ctypes.byref(h)))
        self.h = h

    def halo_init(self, unique_id: bytes, rank: int, nranks: int):
        """Join the NCCL slab exchange (collective over the nranks processes)."""
        _prefer_torch_nccl()
        _check(lib().r3d_gpu_halo_init(self.h, unique_id, len(unique_id), rank, nranks))

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            lib().r3d_gpu_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def upload(self, st: HostState):
        sc = Scalars(**{k: (int(v) if k == "nit" else v) for k, v in st.scalars.items()})
        c = st._c()
        _check(lib().r3d_gpu_upload(self.h, ctypes.byref(c), ctypes.byref(sc)))

    def download(self, st: HostState) -> Dict[str, float]:
        sc = Scalars()
        c = st._c()
        _check(lib().r3d_gpu_download(self.h, ctypes.byref(c), ctypes.byref(sc)))
        st.scalars = sc.as_dict()
        return st.scalars

    def step(self, nstages: int = 3) -> Dict[str, float]:
        sc = Scalars()
        _check(lib().r3d_gpu_step(self.h, nstages, ctypes.byref(sc)))
        return sc.as_dict()

    def run(self, nsteps: int) -> Dict[str, float]:
        sc = Scalars()
        _check(lib().r3d_gpu_run(self.h, nsteps, ctypes.byref(sc)))
        return sc.as_dict()

    def enqueue(self, nsteps: int):
        _check(lib().r3d_gpu_enqueue(self.h, nsteps))

    def run_timed(self, nsteps: int):
        sc, tm = Scalars(), Timing()
        _check(lib().r3d_gpu_run_timed(self.h, nsteps, ctypes.byref(sc), ctypes.byref(tm)))
        return sc.as_dict(), {n: getattr(tm, n) for n, _ in tm._fields_}

    def totals(self):
        m, e = ctypes.c_double(), ctypes.c_double()
        _check(lib().r3d_gpu_totals(self.h, ctypes.byref(m), ctypes.byref(e)))
        return m.value, e.value

    def setup(self) -> Dict[str, float]:
        """Build the initial state on the device (r3d_gpu_setup): the same state as
        upload(HostState.setup(p)), without host 3D arrays; returns the scalars."""
        sc = Scalars()
        _check(lib().r3d_gpu_setup(self.h, ctypes.byref(sc)))
        return sc.as_dict()

    def accumulators(self) -> Dict[str, np.ndarray]:
        """The RK accumulators zru .. ztt (+ zbx zby zbz), shapes (NZ, NY, NX), interior cells."""
        NX, NY, NZ = dims(self.p)
        if self.slab is not None:
            NZ = self.slab[1] + 2
        names = ["zru", "zrv", "zrw", "zro", "ztt"] + (["zbx", "zby", "zbz"] if self.p.lmag else [])
        out = {n: np.zeros((NZ, NY, NX)) for n in names}
        ptrs = (ctypes.c_void_p * 8)(*([out[n].ctypes.data for n in names] + [None] * (8 - len(names))))
        _check(lib().r3d_gpu_download_accumulators(self.h, ptrs))
        return out

    def compare(self, ref: "GpuSim") -> Dict[str, Dict[str, float]]:
        """Error of this state against ref's, on the device: per field rel_l2 =
        ||self - ref|| / ||ref|| and rel_linf = max|self - ref| / max|ref| over the interior."""
        names = ["ru", "rv", "rw", "ro", "tt"] + (["bx", "by", "bz"] if self.p.lmag else [])
        out = np.zeros(4 * len(names))
        _check(lib().r3d_gpu_compare(self.h, ref.h, out.ctypes.data))
        res = {}
        for q, n in enumerate(names):
            sd, sr, md, mr = out[4 * q:4 * q + 4]
            res[n] = {"rel_l2": float(np.sqrt(sd) / np.sqrt(sr)) if sr > 0 else float(np.sqrt(sd)),
                      "rel_linf": float(md / mr) if mr > 0 else float(md)}
        return res

    def fluxes(self) -> Dict[str, np.ndarray]:
        """FLUXES of the current state: fu fv fw fr ft (+ w1 w2 w3), shapes (NZ, NY, NX)."""
        NX, NY, NZ = dims(self.p)
        if self.slab is not None:
            NZ = self.slab[1] + 2
        names = ["fu", "fv", "fw", "fr", "ft"] + (["w1", "w2", "w3"] if self.p.lmag else [])
        out = {n: np.zeros((NZ, NY, NX)) for n in names}
        dp = ctypes.POINTER(ctypes.c_double)
        arr = (dp * len(names))(*[out[n].ctypes.data_as(dp) for n in names])
        _check(lib().r3d_gpu_fluxes(self.h, arr))
        return out

    def work(self, fluxes: bool = True) -> Dict[str, np.ndarray]:
        """The FLUXES work arrays of a gstate dump after a full step: uu vv ww of the third stage's
        input (+ fu fv fw fr ft unless fluxes=False), shapes (NZ, NY, NX)."""
        NX, NY, NZ = dims(self.p)
        if self.slab is not None:
            NZ = self.slab[1] + 2
        names = ["uu", "vv", "ww", "fu", "fv", "fw", "fr", "ft"]
        out = {n: np.zeros((NZ, NY, NX)) for n in names[:8 if fluxes else 3]}
        dp = ctypes.POINTER(ctypes.c_double)
        arr = (dp * 8)(*[out[n].ctypes.data_as(dp) if n in out else dp() for n in names])
        _check(lib().r3d_gpu_download_work(self.h, arr))
        return out

    def debug_tma_extra(self, nbytes: int):
        """Test hook: make the stage kernels' bounded TMA waits run out (0 switches it off)."""
        _check(lib().r3d_gpu_debug_tma_extra(self.h, nbytes))

    def debug_dt_filter(self, margin: float = float("nan")) -> int:
        """Test hook of the third stage's dt filter: set its relative margin (NaN: unchanged; < 0
        forces a full re-evaluation every step) and return the re-evaluations since the upload."""
        n = ctypes.c_int(0)
        _check(lib().r3d_gpu_debug_dt_filter(self.h, margin, ctypes.byref(n)))
        return n.value

    # ---- discrete adjoint (FP64) ----
    def _fields(self):
        return FIELDS3D if self.p.lmag else FIELDS3D[:5]

    def _adjoint_call(self, fn, seed: Dict[str, np.ndarray]) -> Dict[str, np.ndarray]:
        NX, NY, NZ = dims(self.p)
        if self.slab is not None:
            NZ = self.slab[1] + 2
        names = self._fields()
        dp = ctypes.POINTER(ctypes.c_double)
        src = [np.ascontiguousarray(seed[n], dtype=np.float64).reshape(NZ, NY, NX) for n in names]
        out = {n: np.zeros((NZ, NY, NX)) for n in names}
        sp = (dp * len(names))(*[a.ctypes.data_as(dp) for a in src])
        gp = (dp * len(names))(*[out[n].ctypes.data_as(dp) for n in names])
        _check(fn(self.h, sp, gp))
        return out

    def adjoint_record(self, nsteps: int, checkpoint_every: int) -> Dict[str, float]:
        """Run nsteps forward (as run()) keeping a checkpoint every checkpoint_every steps."""
        sc = Scalars()
        _check(lib().r3d_gpu_adjoint_record(self.h, nsteps, checkpoint_every, ctypes.byref(sc)))
        return sc.as_dict()

    def adjoint_backward(self, seed: Dict[str, np.ndarray]) -> Dict[str, np.ndarray]:
        """Cotangent of the recorded start state from the cotangent of the recorded final state."""
        return self._adjoint_call(lib().r3d_gpu_adjoint_backward, seed)

    def adjoint_step(self, seed: Dict[str, np.ndarray]) -> Dict[str, np.ndarray]:
        """One-step vector-Jacobian product at the current state (the state is not advanced)."""
        return self._adjoint_call(lib().r3d_gpu_adjoint_step, seed)

    @property
    def adjoint_memory_bytes(self) -> int:
        b = ctypes.c_int64()
        _check(lib().r3d_gpu_adjoint_memory(self.h, ctypes.byref(b)))
        return int(b.value)

    @property
    def stream(self) -> int:
        return int(lib().r3d_gpu_stream(self.h) or 0)

    @property
    def memory_bytes(self) -> int:
        b = ctypes.c_int64()
        _check(lib().r3d_gpu_memory(self.h, ctypes.byref(b)))
        return int(b.value)


def _prefer_torch_nccl():
    """In a process that uses PyTorch, load torch (and with it its NCCL) before the library
    opens NCCL, so both use the same NCCL."""
    try:
        import torch  # noqa: F401
    except ImportError:
        pass


def nccl_unique_id() -> bytes:
    """128-byte NCCL id for r3d_gpu_halo_init (rank 0 makes it, every rank receives it)."""
    _prefer_torch_nccl()
    buf = ctypes.create_string_buffer(128)
    _check(lib().r3d_nccl_unique_id(buf, 128))
    return buf.raw


class GpuMesh:
    """The z-slab decomposition inside one process (r3d_mesh_*): nslabs slabs on one device."""

    def __init__(self, p: Params, nslabs: int):
        self.p = p
        h = ctypes.c_void_p()
        _check(lib().r3d_mesh_create(ctypes.byref(p), nslabs, ctypes.byref(h)))
        self.h = h
        self.nslabs = nslabs

    def slab(self, r: int):
        z0, nz = ctypes.c_int(), ctypes.c_int()
        _check(lib().r3d_mesh_slab(self.h, r, ctypes.byref(z0), ctypes.byref(nz)))
        return z0.value, nz.value

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            lib().r3d_mesh_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def upload(self, st: HostState):
        sc = Scalars(**{k: (int(v) if k == "nit" else v) for k, v in st.scalars.items()})
        c = st._c()
        _check(lib().r3d_mesh_upload(self.h, ctypes.byref(c), ctypes.byref(sc)))

    def step(self, nstages: int = 3) -> Dict[str, float]:
        sc = Scalars()
        _check(lib().r3d_mesh_step(self.h, nstages, ctypes.byref(sc)))
        return sc.as_dict()

    def debug_dt_filter(self, margin: float = float("nan")) -> int:
        """Test hook: the dt-filter margin of every slab (NaN: unchanged); returns the refolds
        of all slabs since the upload."""
        n = ctypes.c_int(0)
        _check(lib().r3d_mesh_debug_dt_filter(self.h, margin, ctypes.byref(n)))
        return n.value

    def run(self, nsteps: int) -> Dict[str, float]:
        sc = Scalars()
        _check(lib().r3d_mesh_run(self.h, nsteps, ctypes.byref(sc)))
        return sc.as_dict()

    def download(self, st: HostState) -> Dict[str, float]:
        sc = Scalars()
        c = st._c()
        _check(lib().r3d_mesh_download(self.h, ctypes.byref(c), ctypes.byref(sc)))
        st.scalars = sc.as_dict()
        return st.scalars


def version() -> str:
    return lib().r3d_version().decode()
