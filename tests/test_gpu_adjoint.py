"""Discrete adjoint of the FP64 RK3 step on the GPU (r3d_gpu_adjoint_*).

The reference has no adjoint; the checks are against the forward map itself:

* dot-product tests <lambda, J V> = <J^T lambda, V>, with J V the exact tangent of the numpy
  restatement of the step (oracle/tangent_np.py run with complex arrays, "complex step") and
  J^T lambda from the GPU: one step, and a checkpointed multi-step run whose segments are
  recomputed (hydro and MHD, rotation, the three branches of the dt minimum);
* the adjoint benchmark case: MHD 64x64x128 (--beta 10 --rm 1, magnetic layer ampb 0.1 with the
  bfh 2 / bzp 20 shape of the MHD benchmark grid, since the reference defaults bfh = bzp = 0 give
  an empty layer), RAN2 seed 5, 200 RK3 steps with a checkpoint every 20: the gradient of the
  final volume-integrated kinetic energy w.r.t. the initial temperature field, through the
  torch.autograd.Function, against central differences of the forward in 8 random unit
  directions (<= 1e-6 relative); the +-eps runs of one direction repeated on the CPU
  restatement of the reference (r3d_oracle.c) give bit-identical energies;
* refusals: FP32-bulk and a time-dependent plume boundary.
"""
import numpy as np
import pytest

import r3d_b200 as R
from oracle import Oracle
from tangent_np import NumpyStep

MAG = ["--lmag", "1", "--beta", "10", "--rm", "1", "--ampb", "0.1", "--bfh", "2", "--bzp", "20"]
I3 = (slice(1, -1), slice(1, -1), slice(1, -1))


def names_of(p):
    return R.FIELDS3D if p.lmag else R.FIELDS3D[:5]


def periodic(a):
    a[:, 0, :] = a[:, -2, :]
    a[:, -1, :] = a[:, 1, :]
    a[:, :, 0] = a[:, :, -2]
    a[:, :, -1] = a[:, :, 1]
    return a


def interior_dot(A, B, names):
    return sum(float(np.sum(A[n][I3] * B[n][I3])) for n in names)


def state_after(p, presteps):
    st = R.HostState.setup(p)
    with R.GpuSim(p) as sim:
        sim.upload(st)
        if presteps:
            sim.run(presteps)
        sim.download(st)
    return st


def tangent(flags, seed, X, V, nsteps):
    """Exact J V of nsteps steps at X (complex step through the numpy restatement)."""
    ns = NumpyStep(Oracle(flags).init(seed))
    h = 1e-30
    Xc = {n: X[n] + 1j * h * V[n] for n in ns.fields}
    Xc, _ = ns.run(Xc, nsteps)
    return {n: Xc[n].imag / h for n in ns.fields}


def random_pair(p, rng):
    NX, NY, NZ = R.dims(p)
    V, lam = {}, {}
    for n in names_of(p):
        v = np.zeros((NZ, NY, NX))
        v[I3] = rng.standard_normal((NZ - 2, NY - 2, NX - 2))
        V[n] = periodic(v)
        l_ = np.zeros((NZ, NY, NX))
        l_[I3] = rng.standard_normal((NZ - 2, NY - 2, NX - 2))
        lam[n] = l_
    return V, lam


DOT_CASES = [
    ("hydro", ["--npx", "16", "--npy", "12", "--npz", "24"], 3, 2),
    ("mhd", ["--npx", "16", "--npy", "12", "--npz", "24"] + MAG, 5, 2),
    ("rotation_flux_bottom", ["--npx", "12", "--npy", "10", "--npz", "16", "--lrot", "1", "--ry", "2", "--ang",
                              "0.4", "--izcon", "1", "--itcon", "0"], 7, 1),
    ("cfl_limited", ["--npx", "12", "--npy", "10", "--npz", "16", "--re", "1000", "--pr", "1"], 3, 2),
    ("viscous_limited", ["--npx", "12", "--npy", "10", "--npz", "16", "--re", "0.1", "--pr", "100"], 3, 2),
]


@pytest.mark.gpu
@pytest.mark.parametrize("name,flags,seed,pre", DOT_CASES, ids=[c[0] for c in DOT_CASES])
def test_adjoint_step_dot_product(name, flags, seed, pre):
    p = R.parse(flags + ["--seed", str(seed)])
    st = state_after(p, pre)
    X = {n: st.fields[n].copy() for n in names_of(p)}
    rng = np.random.default_rng(seed)
    for _ in range(2):
        V, lam = random_pair(p, rng)
        JV = tangent(flags, seed, X, V, 1)
        with R.GpuSim(p) as sim:
            sim.upload(st)
            g = sim.adjoint_step(lam)
        lhs = interior_dot(lam, JV, names_of(p))
        rhs = interior_dot(g, V, names_of(p))
        assert abs(lhs - rhs) <= 1e-11 * abs(lhs), (lhs, rhs)
        for n in names_of(p):  # gradients live on interior cells only
            gg = g[n].copy()
            gg[I3] = 0.0
            assert not gg.any()


@pytest.mark.gpu
@pytest.mark.parametrize("mhd", [False, True], ids=["hydro", "mhd"])
def test_adjoint_checkpointed_trajectory(mhd):
    """7 steps, checkpoint every 3: segments of 3, 3 and 1 steps recomputed in reverse."""
    flags = ["--npx", "16", "--npy", "12", "--npz", "24"] + (MAG if mhd else [])
    seed = 11
    p = R.parse(flags + ["--seed", str(seed)])
    st = state_after(p, 2)
    X = {n: st.fields[n].copy() for n in names_of(p)}
    V, lam = random_pair(p, np.random.default_rng(3))
    JV = tangent(flags, seed, X, V, 7)
    with R.GpuSim(p) as sim:
        sim.upload(st)
        sim.adjoint_record(7, 3)
        g = sim.adjoint_backward(lam)
        assert sim.adjoint_memory_bytes > 0
    lhs = interior_dot(lam, JV, names_of(p))
    rhs = interior_dot(g, V, names_of(p))
    assert abs(lhs - rhs) <= 1e-11 * abs(lhs), (lhs, rhs)


def kinetic_energy_np(fields, dV):
    ru, rv, rw, ro = (fields[n][I3] for n in ("ru", "rv", "rw", "ro"))
    return float(np.sum(0.5 * (ru * ru + rv * rv + rw * rw) / ro * dV))


def volume_weights(st, p):
    """Cell volumes of the stretched grid: 1/(2 h dxxdx) per direction."""
    hx, hy, hz = (R.derived(p, n) for n in ("hx", "hy", "hz"))
    wx = 1.0 / (2.0 * hx * st.lines["dxxdx"][1:-1])
    wy = 1.0 / (2.0 * hy * st.lines["dyydy"][1:-1])
    wz = 1.0 / (2.0 * hz * st.lines["dzzdz"][1:-1])
    return wz[:, None, None] * wy[None, :, None] * wx[None, None, :]


ADJ_FLAGS = ["--npx", "64", "--npy", "64", "--npz", "128"] + MAG
ADJ_SEED, ADJ_STEPS, ADJ_EVERY = 5, 200, 20


@pytest.mark.gpu
def test_adjoint_kinetic_energy_gradient_vs_central_differences():
    import torch
    from r3d_b200.autograd import RK3Trajectory, stack

    p = R.parse(ADJ_FLAGS + ["--seed", str(ADJ_SEED)])
    base = R.HostState.setup(p)
    dV = volume_weights(base, p)
    names = names_of(p)
    q_tt = names.index("tt")
    sim = R.GpuSim(p)
    try:
        x0 = stack(base, p).clone().requires_grad_(True)
        xN = RK3Trajectory.apply(x0, sim, base, ADJ_STEPS, ADJ_EVERY)
        dVt = torch.from_numpy(dV)
        ru, rv, rw, ro = (xN[names.index(n)][I3] for n in ("ru", "rv", "rw", "ro"))
        J = (0.5 * (ru * ru + rv * rv + rw * rw) / ro * dVt).sum()
        J.backward()
        grad_T = x0.grad[q_tt].numpy()
        assert not np.any(grad_T[:, 0, :]) and not np.any(grad_T[0])  # ghosts carry no gradient

        def energy(theta):
            st = base.copy()
            st.fields["tt"] = periodic(st.fields["tt"] + theta)
            sim.upload(st)
            sim.run(ADJ_STEPS)
            sim.download(st)
            return kinetic_energy_np(st.fields, dV)

        J0 = energy(0.0)
        assert J0 == pytest.approx(float(J.detach()), rel=1e-13)  # the recorded run is the plain run
        rng = np.random.default_rng(2024)
        # The directional derivative along a unit direction is ~1e-4 of J, so the rounding noise of
        # J (~1e-14 relative after 200 steps) divided by eps dominates the difference below
        # eps ~ 1e-4, and the O(eps^2) truncation error above ~3e-3; eps = 1e-3 sits between
        # (differences agree with the adjoint to ~1e-8 there).
        eps = 1e-3
        worst = 0.0
        dirs = []
        for _ in range(8):
            d = np.zeros_like(base.fields["tt"])
            d[I3] = rng.standard_normal(d[I3].shape)
            d /= np.linalg.norm(d[I3])
            d = periodic(d)
            dirs.append(d)
            jp, jm = energy(eps * d), energy(-eps * d)
            fd = (jp - jm) / (2.0 * eps)
            ad = float(np.sum(grad_T[I3] * d[I3]))
            worst = max(worst, abs(ad - fd) / abs(fd))
        assert worst <= 1e-6, worst
    finally:
        sim.close()

    # the same directional difference from the CPU restatement of the reference: identical J
    d = dirs[0]
    for sgn in (1.0, -1.0):
        o = Oracle(ADJ_FLAGS).init(ADJ_SEED)
        tt = o.field("tt")
        tt[...] = periodic(tt + sgn * eps * d)
        for _ in range(ADJ_STEPS):
            o.step()
        gpu_j = energy_on_gpu(p, base, sgn * eps * d)
        cpu_j = kinetic_energy_np({n: o.field(n) for n in ("ru", "rv", "rw", "ro")}, dV)
        assert cpu_j == gpu_j


def energy_on_gpu(p, base, theta):
    st = base.copy()
    st.fields["tt"] = periodic(st.fields["tt"] + theta)
    with R.GpuSim(p) as sim:
        sim.upload(st)
        sim.run(ADJ_STEPS)
        sim.download(st)
    return kinetic_energy_np(st.fields, volume_weights(base, p))


@pytest.mark.gpu
def test_adjoint_refusals():
    p = R.parse(["--npx", "16", "--npy", "12", "--npz", "24", "--precision", "fp32bulk"])
    st = R.HostState.setup(p)
    with R.GpuSim(p) as sim:
        sim.upload(st)
        with pytest.raises(R.R3dError) as e:
            sim.adjoint_record(2, 1)
        assert e.value.code == R.R3D_EINVAL
    p = R.parse(["--npx", "16", "--npy", "12", "--npz", "24", "--tc", "0.5"])
    st = R.HostState.setup(p)
    with R.GpuSim(p) as sim:
        sim.upload(st)
        with pytest.raises(R.R3dError) as e:
            sim.adjoint_step({n: np.zeros_like(st.fields[n]) for n in names_of(p)})
        assert e.value.code == R.R3D_EINVAL
        with pytest.raises(R.R3dError) as e:
            sim.adjoint_backward({n: np.zeros_like(st.fields[n]) for n in names_of(p)})
        assert e.value.code == R.R3D_ESTATE
