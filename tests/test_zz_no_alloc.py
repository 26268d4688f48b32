"""The allocation-free time-step limits (r3d_dt_limits_noalloc) against the regular step.

Some callers cannot call cudaMalloc: a program that reserves the GPU's memory in its own pool
up front, or a time loop that must not pay the synchronisation an allocation may imply.  For
them r3d_dt_limits_noalloc computes {dt, umach} of a state they already hold in device memory,
keeping its partial results in a fixed file-scope device array instead of allocated scratch.

Here the "caller" owns the state in device memory (torch tensors); two calls in a row (the
uploaded state, then the state after one step) must give exactly the dt and umach that the
existing entry point r3d_gpu_step reports for the same state: hydro with constant and with
variable conductivity, MHD (the field's b2 term in the fast-mode speed and the magnetic
diffusion limit), on the legacy default stream and on a caller's own stream.  This file is
collected last, so a run that stops at the first failure has run every other test before it.
"""
import ctypes

import numpy as np
import pytest

import r3d_b200 as R

MAG = ["--lmag", "1", "--beta", "10", "--rm", "1", "--ampb", "0.1", "--bfh", "2", "--bzp", "20"]
CASES = {
    "hydro": ["--npx", "40", "--npy", "24", "--npz", "48", "--seed", "9"],
    "variable_kappa": ["--npx", "24", "--npy", "20", "--npz", "36", "--pzp", "0.5", "--sigma", "0.1",
                       "--polys", "1.5", "--seed", "7"],
    "mhd": ["--npx", "24", "--npy", "20", "--npz", "40", "--seed", "7"] + MAG,
}


def _noalloc(p, fields, lines, out_ptr, stream=None):
    f = R.lib().r3d_dt_limits_noalloc
    f.argtypes = [ctypes.POINTER(R.Params), ctypes.POINTER(ctypes.c_void_p),
                  ctypes.POINTER(ctypes.c_void_p), ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    fa = (ctypes.c_void_p * 8)(*fields)
    la = (ctypes.c_void_p * 4)(*lines)
    return f(ctypes.byref(p), fa, la, out_ptr, stream)


@pytest.mark.parametrize("npx,npy", [(20000, 20000), (32, 8 * 65535 + 1)])
def test_noalloc_rejects_grids_beyond_its_fixed_array(npx, npy):
    """Sizes beyond the fixed partials array, or beyond a launch's 65535 tile rows, are refused
    with R3D_EINVAL before any GPU work."""
    p = R.parse(["--npx", str(npx), "--npy", str(npy), "--npz", "64"])
    rc = _noalloc(p, [1] * 8, [1] * 4, 1)
    assert rc == R.R3D_EINVAL
    assert "too large" in R.lib().r3d_last_error().decode()


@pytest.mark.gpu
@pytest.mark.parametrize("case", sorted(CASES))
@pytest.mark.parametrize("on_stream", [False, True], ids=["default_stream", "own_stream"])
def test_noalloc_dt_matches_step_on_two_calls(case, on_stream):
    import torch

    p = R.parse(CASES[case])
    st = R.HostState.setup(p)
    names = ("ru", "rv", "rw", "ro", "tt", "bx", "by", "bz")[: 8 if p.lmag else 5]
    dev = torch.device("cuda", p.gpu_id)
    stream = torch.cuda.Stream(device=dev) if on_stream else None
    with R.GpuSim(p) as sim:
        sim.upload(st)
        for call in range(2):
            # the caller's own device copy of the current state and metric lines
            fields = [torch.from_numpy(st.fields[n]).to(dev) for n in names]
            lines = [torch.from_numpy(st.lines[n]).to(dev) for n in ("ddx", "ddy", "ddz", "rkapa")]
            out = torch.full((2,), float("nan"), dtype=torch.float64, device=dev)
            torch.cuda.synchronize()
            ptrs = [t.data_ptr() for t in fields] + [None] * (8 - len(fields))
            rc = _noalloc(p, ptrs, [t.data_ptr() for t in lines], out.data_ptr(),
                          stream.cuda_stream if stream is not None else None)
            assert rc == R.R3D_OK, R.lib().r3d_last_error().decode()
            torch.cuda.synchronize()
            dt, umach = out.cpu().numpy().tolist()
            sc = sim.step()  # the existing entry point: dt and umach of the same state
            assert dt == sc["dt"], f"call {call}: dt {dt!r} != step dt {sc['dt']!r}"
            assert umach == sc["umach"], f"call {call}: umach {umach!r} != {sc['umach']!r}"
            assert np.isfinite(dt) and dt > 0.0
            sim.download(st)  # the next call sees the state after this step
