"""Multi-process z-slab runs: partition and the NCCL id hand-out (host plumbing only).

The device side is r3d_gpu_create_slab + r3d_gpu_halo_init (halo.cu): one process per GPU,
rank r holding the r-th slab in z order.  torch.distributed (any backend, gloo included) only
carries the 128-byte NCCL id from rank 0 to the others.
"""
from __future__ import annotations

from typing import Optional, Tuple

from . import nccl_unique_id


def slab_of(npz: int, rank: int, nranks: int) -> Tuple[int, int]:
    """(z0, nz) of rank's slab: npz // nranks planes each, the first npz % nranks one more
    (the split of r3d_mesh_create)."""
    if nranks < 1 or not 0 <= rank < nranks:
        raise ValueError("bad rank / nranks")
    base, extra = divmod(npz, nranks)
    if base < 4:
        raise ValueError("each slab needs at least 4 planes")
    z0 = rank * base + min(rank, extra)
    return z0, base + (1 if rank < extra else 0)


def share_unique_id(rank: int, dist=None, make=nccl_unique_id) -> bytes:
    """Rank 0 makes the id; a torch.distributed module (initialised) broadcasts it."""
    uid = make() if rank == 0 else bytes(128)
    if dist is not None and dist.get_world_size() > 1:
        import torch

        t = torch.tensor(list(uid), dtype=torch.uint8)
        dist.broadcast(t, 0)
        uid = bytes(t.tolist())
    return uid


def open_slab(p, rank: int, nranks: int, dist=None, uid: Optional[bytes] = None):
    """GpuSim over this rank's slab, joined to the others (collective)."""
    from . import GpuSim

    z0, nz = slab_of(p.npz, rank, nranks)
    sim = GpuSim(p, slab=(z0, nz))
    if nranks > 1 or uid is not None:
        sim.halo_init(uid if uid is not None else share_unique_id(rank, dist), rank, nranks)
    return sim, (z0, nz)
