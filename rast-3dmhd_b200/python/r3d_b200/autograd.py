"""torch.autograd bridge for the discrete adjoint of the RK3 step.

``RK3Trajectory.apply(x0, sim, base, nsteps, every)`` is the map X_0 -> X_N of nsteps FP64 RK3
steps on the GPU (r3d_gpu_adjoint_record); its backward is r3d_gpu_adjoint_backward, the
hand-written reverse sweep with a state checkpoint every ``every`` steps and recomputation in
between.  States are float64 CPU tensors shaped (nfields, NZ, NY, NX) in the host layout of
HostState (fields ru rv rw ro tt, + bx by bz with lmag).  The x/y ghost cells of x0 are
replaced by the periodic images of its interior before the run, so the map depends on the
interior only and the gradient's ghost entries are 0; the z ghost planes are constants.

    sim = r3d_b200.GpuSim(p); base = r3d_b200.HostState.setup(p)
    x0 = stack(base).requires_grad_()
    xN = RK3Trajectory.apply(x0, sim, base, 200, 20)
    kinetic_energy(xN).backward()          # x0.grad = dJ/dX_0
"""
from __future__ import annotations

import numpy as np
import torch

from . import FIELDS3D, GpuSim, HostState


def field_names(p) -> list:
    return FIELDS3D if p.lmag else FIELDS3D[:5]


def periodic_ghosts(a: np.ndarray) -> np.ndarray:
    """x/y ghost cells of every plane set to the periodic images of the interior (in place)."""
    a[:, 0, :] = a[:, -2, :]
    a[:, -1, :] = a[:, 1, :]
    a[:, :, 0] = a[:, :, -2]
    a[:, :, -1] = a[:, :, 1]
    return a


def stack(st: HostState, p) -> torch.Tensor:
    return torch.from_numpy(np.stack([st.fields[n] for n in field_names(p)]))


class RK3Trajectory(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x0: torch.Tensor, sim: GpuSim, base: HostState, nsteps: int, every: int):
        names = field_names(sim.p)
        st = base.copy()
        x = x0.detach().cpu().numpy()
        for q, n in enumerate(names):
            st.fields[n][...] = periodic_ghosts(np.array(x[q], dtype=np.float64))
        sim.upload(st)
        ctx.scalars = sim.adjoint_record(nsteps, every)
        sim.download(st)
        ctx.sim = sim
        return torch.from_numpy(np.stack([st.fields[n] for n in names]))

    @staticmethod
    def backward(ctx, g: torch.Tensor):
        names = field_names(ctx.sim.p)
        gn = g.detach().cpu().numpy()
        grad = ctx.sim.adjoint_backward({n: gn[q] for q, n in enumerate(names)})
        return torch.from_numpy(np.stack([grad[n] for n in names])), None, None, None, None
