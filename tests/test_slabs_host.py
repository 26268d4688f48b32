"""Host side of the z-slab decomposition: slab set-up, partition, and the NCCL id hand-out over
a two-process gloo group (no GPU needed)."""
import os

import numpy as np
import pytest

import r3d_b200 as R
from r3d_b200 import dist as D

MAG = ["--lmag", "1", "--beta", "10", "--rm", "1", "--ampb", "0.1", "--bfh", "2", "--bzp", "20"]


@pytest.mark.parametrize("mhd", [False, True], ids=["hydro", "mhd"])
def test_setup_slab_equals_global_slices(mhd):
    p = R.parse(["--npx", "12", "--npy", "10", "--npz", "24", "--seed", "5"] + (MAG if mhd else []))
    g = R.HostState.setup(p)
    for z0, nz in ((0, 6), (6, 7), (13, 11), (0, 24), (5, 19)):
        sl = R.HostState.setup_slab(p, z0, nz)
        v = g.slab_view(z0, nz)
        for n in sl.fields:
            assert np.array_equal(sl.fields[n], v.fields[n]), (z0, nz, n)
        for n in sl.lines:
            assert np.array_equal(sl.lines[n], v.lines[n]), (z0, nz, n)
        assert sl.scalars == g.scalars


def test_slab_partition():
    for npz in (8, 24, 37, 512):
        for n in (1, 2, 3, 4):
            if npz // n < 4:
                with pytest.raises(ValueError):
                    D.slab_of(npz, 0, n)
                continue
            parts = [D.slab_of(npz, r, n) for r in range(n)]
            assert parts[0][0] == 0 and sum(nz for _, nz in parts) == npz
            for (a, na), (b, _) in zip(parts, parts[1:]):
                assert a + na == b
    with pytest.raises(R.R3dError):
        R.HostState.setup_slab(R.parse(["--npx", "8", "--npy", "8", "--npz", "8"]), 6, 4)


def _rank(rank, world, port, q):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        uid = D.share_unique_id(rank, dist, make=lambda: bytes(range(128)))
        z0, nz = D.slab_of(40, rank, world)
        q.put((rank, uid, z0, nz))
    finally:
        dist.destroy_process_group()


def test_unique_id_broadcast_two_ranks():
    import multiprocessing as mp
    import socket

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    out = sorted(q.get(timeout=120) for _ in range(2))
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    assert out[0][1] == out[1][1] == bytes(range(128))
    assert (out[0][2], out[0][3], out[1][2], out[1][3]) == (0, 20, 20, 20)


def test_nccl_unique_id_is_128_bytes():
    uid = R.nccl_unique_id()
    assert isinstance(uid, bytes) and len(uid) == 128


def _slab_rank(rank, world, port, q, flags, seed, nsteps):
    """One rank of the multi-process z-slab step on the CPU: the numpy restatement of the step on
    this rank's slab, ghost planes swapped with the z neighbours after every stage and the dt
    minimum all-reduced before every step - the protocol the NCCL path runs on GPUs."""
    import numpy as np
    import torch
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle import Oracle
        from tangent_np import NumpyStep

        o = Oracle(flags).init(seed)
        full = NumpyStep(o)
        X0 = {n: o.field(n).copy() for n in full.fields}
        z0, nz = D.slab_of(full.npz, rank, world)
        s = full.slab(z0, nz)

        def reduce_min(x):
            t = torch.tensor([x], dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MIN)
            return float(t.item())

        def exchange(X):
            reqs, recv = [], []
            for n in s.fields:
                a = X[n]
                if rank > 0:    # my first plane up, the slab above's last plane into my plane 0
                    reqs.append(dist.isend(torch.from_numpy(a[1].copy()), rank - 1))
                    recv.append((n, 0, torch.empty(a[0].shape, dtype=torch.float64), rank - 1))
                if rank < world - 1:
                    reqs.append(dist.isend(torch.from_numpy(a[nz].copy()), rank + 1))
                    recv.append((n, nz + 1, torch.empty(a[0].shape, dtype=torch.float64), rank + 1))
            for n, k, t, src in recv:
                dist.recv(t, src)
                X[n][k] = t.numpy()
            for r in reqs:
                r.wait()

        s.reduce_min, s.exchange = reduce_min, exchange
        X = {n: a[z0:z0 + nz + 2].copy() for n, a in X0.items()}
        Xs, dts = s.run(X, nsteps)
        Xf, dtf = full.run(X0, nsteps)       # the single domain, for comparison
        same = all(np.array_equal(Xs[n][1:-1, 1:-1, 1:-1], Xf[n][z0 + 1:z0 + nz + 1, 1:-1, 1:-1]) for n in s.fields)
        q.put((rank, same, dts == dtf, s.top, s.bot))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("flags,world", [
    (["--npx", "12", "--npy", "10", "--npz", "16"], 2),
    (["--npx", "10", "--npy", "8", "--npz", "20", "--lmag", "1", "--beta", "10", "--rm", "1", "--ampb", "0.1",
      "--bfh", "2", "--bzp", "20"], 3),
], ids=["hydro_2ranks", "mhd_3ranks"])
def test_multirank_slab_protocol_equals_single_domain(flags, world):
    """gloo ranks on the CPU run the z-slab decomposition (exchange after each stage, dt
    all-reduce per step) and reproduce the single-domain step bit for bit."""
    import multiprocessing as mp
    import socket

    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_slab_rank, args=(r, world, port, q, flags, 5, 3)) for r in range(world)]
    for pr in procs:
        pr.start()
    out = sorted(q.get(timeout=300) for _ in range(world))
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    assert all(o[1] for o in out), out
    assert all(o[2] for o in out), out
    assert out[0][3] and not out[0][4] and out[-1][4] and not out[-1][3]


def test_missing_nccl_is_a_clear_error():
    """Without an NCCL to load, the slab transport fails with a status and a message (no abort):
    a fresh process, nothing loaded NCCL before, R3D_NCCL_LIBRARY pointing at nothing."""
    import subprocess
    import sys

    code = (
        "import ctypes, sys\n"
        "sys.path.insert(0, %r)\n"
        "import r3d_b200 as R\n"
        "L = R.lib()\n"
        "buf = ctypes.create_string_buffer(128)\n"
        "rc = L.r3d_nccl_unique_id(buf, 128)\n"
        "print(rc, R.lib().r3d_last_error().decode())\n"
    ) % os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "rast-3dmhd_b200", "python")
    env = dict(os.environ, R3D_NCCL_LIBRARY="/nonexistent/libnccl-missing.so")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=120, env=env)
    assert r.returncode == 0, r.stderr
    rc, msg = r.stdout.split(" ", 1)
    assert int(rc) != 0 and "NCCL is not available" in msg, r.stdout
