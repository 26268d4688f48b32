"""Benchmark: Rast-3DMHD FP64 RK3 step on B200, in Mcell-updates/s.

Workload (one "step" = one full RK3 time step, dt reduction, BCON and ghost fill included):
FP64 hydro on the 504 x 504 x 512 grid with default physics (re=2 pr=0.05 theta=0.25
grav=0.625 gamma=5/3 sff=0.315, ngrid=1, plume top BC), polytropic static IC with the RAN2
temperature perturbation (amplitude 0.005) drawn with seed 3.  Inputs are synthetic (no
dataset exists for this path); the working set (15 x 1.07 GB) is far larger than L2.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Timing: W untimed steps, then K steps timed with CUDA events recorded by the library on the
stream its kernels run on (every launch is bracketed, which also yields the per-kernel
durations for the roofline); barrier + device synchronise on both sides; max over ranks.
With N > 1 (under torchrun, or `--gpus N` alone, which starts the N ranks itself: one process
per GPU, LOCAL_RANK set) the domain grows to 504 x 504 x (512 N) and each rank holds one
504 x 504 x 512 z slab on its GPU (weak scaling): the ghost planes move over NCCL after every
stage and the dt limits are all-reduced on the device every step, inside the timed region.
`--dry-launch` starts the ranks and joins them (gloo) without GPU work: a check of the launch.
The reference arm (--impl reference) times the reference's own CPU sources (compiled
unmodified into oracle/_ref) on the same 504 x 504 x 512 grid, W untimed and K timed steps,
on rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (os.path.join(ROOT, "rast-3dmhd_b200", "python"), os.path.join(ROOT, "oracle")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

GRID = (504, 504, 512)
SEED = 3
FLAGS = ["--npx", str(GRID[0]), "--npy", str(GRID[1]), "--npz", str(GRID[2])]
METRIC = "Mcell-updates/s per RK3 step (FP64, bit-exact vs reference CPU)"
UNIT = "Mcell-updates/s"
# algorithmic HBM bytes per interior cell: stage 1 reads X (5 fields) and writes X', Z'
# (10); stage 2 reads X, Z and writes X', Z' (20); stage 3 reads X, Z and writes X' (15):
# 50 field passes x 8 B per step, i.e. 400 B/cell/step and 400/3 B per cell per stage launch.
BYTES_PER_CELL_STEP = 400.0
BYTES_PER_CELL_STAGE = BYTES_PER_CELL_STEP / 3.0
PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0
TRAFFIC_FILE = os.path.join(ROOT, "profiles", "traffic_stage_fp64_504x504x124_k62.md")


def peak_hbm():
    try:
        with open(PEAKS_FILE) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def stage_traffic_per_launch(cells: int):
    """DRAM bytes per stage launch from the committed ncu summary (scaled by cells), or None."""
    try:
        with open(TRAFFIC_FILE) as f:
            for line in f:
                if line.startswith("traffic_bytes_per_cell_per_stage_launch:"):
                    return float(line.split(":", 1)[1]) * cells
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def wait_first(self, limit_s: float = 5.0):
        """Block until nvidia-smi has produced a sample (it takes a moment to start), then drop
        the samples taken so far so that the summary covers the timed region only."""
        t0 = time.perf_counter()
        while self.proc and not self.lines and time.perf_counter() - t0 < limit_s:
            time.sleep(0.02)
        self.lines = []

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=300))
        pg = dist
    return world, rank, local, pg


def spawn_ranks(n: int) -> int:
    """`bench.py --gpus N` started without a launcher: start the N ranks here, one process per
    GPU (RANK = LOCAL_RANK = r, WORLD_SIZE = N, rendezvous on 127.0.0.1), as torchrun would.
    Rank 0 writes the JSON line to this process's stdout; every rank's log goes to stderr.  A
    rank that fails or does not finish stops the others, and the exit code is nonzero."""
    import socket

    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    limit_s = float(os.environ.get("R3D_BENCH_RANK_TIMEOUT", "3600"))
    procs = []
    for r in range(n):
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE=str(n), LOCAL_WORLD_SIZE=str(n),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, os.path.abspath(__file__)] + sys.argv[1:], env=env,
                                      stdout=_RESULT if r == 0 else sys.stderr, stderr=sys.stderr))
    t0 = time.perf_counter()
    rc = 0
    while any(pr.poll() is None for pr in procs):
        failed = [pr for pr in procs if pr.returncode not in (None, 0)]
        if failed or time.perf_counter() - t0 > limit_s:
            rc = failed[0].returncode if failed else 124
            print(f"bench: rank failed or timed out (rc {rc}); stopping the other ranks", file=sys.stderr)
            for pr in procs:
                if pr.poll() is None:
                    pr.kill()
            break
        time.sleep(0.2)
    for pr in procs:
        pr.wait()
        if pr.returncode != 0 and rc == 0:
            rc = pr.returncode
    return rc


def dry_launch(args, world, rank, pg) -> int:
    """Join the ranks without GPU work: every rank reports its slab of the weak-scaling domain,
    and the 128-byte id a real run hands to the NCCL transport goes from rank 0 to all."""
    from r3d_b200 import dist as D

    npz = GRID[2] * world
    z0, nz = D.slab_of(npz, rank, world)
    uid = D.share_unique_id(rank, pg, make=lambda: bytes(range(128)))
    mine = {"rank": rank, "local_rank": int(os.environ.get("LOCAL_RANK", "0")), "slab": [z0, nz],
            "uid_ok": uid == bytes(range(128))}
    joined = [mine]
    if pg is not None:
        joined = [None] * world
        pg.all_gather_object(joined, mine)
    if rank == 0:
        emit({"dry_launch": True, "n_gpus": world, "requested": args.gpus, "joined": joined,
              "domain": [GRID[0], GRID[1], npz]})
    return 0


def barrier(pg):
    if pg is not None:
        pg.barrier()


def allmax(pg, x: float) -> float:
    if pg is None:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def cpu_reference_sample(warmup: int = 1, nsteps: int = 2):
    """Time the reference CPU sources (or the oracle port when absent) on the benchmark grid
    itself: set-up, `warmup` untimed steps, then `nsteps` timed steps (a bounded sample, about
    15-30 s of host time on 16 threads)."""
    ncores = os.cpu_count() or 1
    args = FLAGS + ["--npey", "1"]
    cells = GRID[0] * GRID[1] * GRID[2]
    try:
        from oracle import Reference

        if not Reference.available():
            raise RuntimeError("reference build absent")
        ranks, threads = reference_layout(ncores)
        _, sec = Reference.time_steps(args, ranks, SEED, warmup, nsteps, threads)
        return {"value": cells * nsteps / sec / 1e6, "unit": UNIT, "cores": ranks * threads,
                "kind": "reference",
                "sample": f"reference CPU sources (src/*.cpp, -O2 -ffp-contract=off -fopenmp) with a "
                          f"thread-rank MPI stand-in, {ranks} ranks x {threads} OpenMP threads, grid "
                          f"{GRID[0]}x{GRID[1]}x{GRID[2]} (the benchmark grid), {warmup} untimed + {nsteps} "
                          f"timed RK3 steps, seed {SEED}, host has {ncores} logical cores"}
    except Exception as e:  # oracle port as the stand-in
        from oracle import Oracle

        o = Oracle(FLAGS).init(SEED)
        for _ in range(warmup):
            o.step()
        t0 = time.perf_counter()
        for _ in range(nsteps):
            o.step()
        sec = time.perf_counter() - t0
        return {"value": cells * nsteps / sec / 1e6, "unit": UNIT, "cores": ncores, "kind": "port",
                "sample": f"C restatement (oracle/r3d_oracle.c, OpenMP) on {GRID[0]}x{GRID[1]}x{GRID[2]}, "
                          f"{nsteps} timed steps ({e})"}


REF_GPU_RANKS = 2  # the reference needs NPEZ >= 2 (src/topology.cpp:50-55)


def reference_gpu_leg(warmup: int = 1, nsteps: int = 3):
    """The reference's own GPU driver (src/gpu.cpp + src/gpu_kernels.cu, unmodified, sm_100a, its
    stock host-staged build) on the benchmark grid: the reference set-up, then `warmup` untimed
    and `nsteps` timed step_gpu calls on two thread-ranks in z sharing this GPU, the device
    synchronised and the ranks joined on both sides (host clock: the driver's own stream is not
    reachable from here)."""
    from oracle import Reference

    cells = GRID[0] * GRID[1] * GRID[2]
    sc, sec = Reference.time_gpu(FLAGS + ["--npey", "1"], REF_GPU_RANKS, SEED, warmup, nsteps)
    return {"value": cells * nsteps / sec / 1e6, "unit": UNIT, "ms_per_step": sec / nsteps * 1e3,
            "steps": nsteps, "warmup": warmup, "final_dt": sc["dt"], "ranks": REF_GPU_RANKS}


def reference_gpu_run(fp64_ms_per_step, limit_s: float = 600.0):
    """reference_gpu_leg in a child process (the driver exits its process on a CUDA error,
    src/gpu.cpp:117-126), set beside the fused FP64 step."""
    from oracle import Reference

    if not Reference.gpu_available():
        return {"unavailable": "reference GPU driver not built (the reference tree was absent at build time)"}
    t0 = time.perf_counter()
    try:
        r = subprocess.run([sys.executable, os.path.abspath(__file__), "--reference-gpu-leg"],
                           capture_output=True, text=True, timeout=limit_s)
    except subprocess.TimeoutExpired:
        return {"unavailable": f"reference GPU leg did not finish within {limit_s:.0f} s"}
    lines = [x for x in r.stdout.splitlines() if x.startswith("{")]
    if r.returncode != 0 or not lines:
        tail = (r.stderr.strip().splitlines() or ["no output"])[-1]
        return {"unavailable": f"reference GPU leg failed (rc {r.returncode}): {tail[:200]}"}
    out = json.loads(lines[-1])
    out["fused_fp64_speedup"] = out["ms_per_step"] / fp64_ms_per_step
    out["wall_s"] = time.perf_counter() - t0
    out["note"] = (f"the reference's stock GPU build (host-staged halos, host-side dt minimum: four "
                   f"whole arrays copied to the host per step, src/gpu.cpp:787-823), its set-up and "
                   f"grid {GRID[0]}x{GRID[1]}x{GRID[2]} seed {SEED}, {REF_GPU_RANKS} thread-ranks in z "
                   f"on this GPU, host clock around synchronised steps; the NCCL build "
                   f"(R3D_COMM_NCCL) needs one GPU per rank")
    return out


def side_run(R, flags, steps, warmup, bytes_per_cell, fp64_ms_per_step):
    """Timed run of another form of the step (same protocol as the headline, events on the
    library stream); returns Mcell-updates/s, % of the HBM roofline by its own algorithmic bytes
    and, for FP32-bulk, the speed-up over the FP64 headline run."""
    p = R.parse(flags)
    npx, npy, npz = p.npx, p.npy, p.npz
    st = R.HostState.setup(p)
    with R.GpuSim(p) as sim:
        sim.upload(st)
        sim.run(warmup)
        _, tm = sim.run_timed(steps)
    cells = npx * npy * npz
    ms = tm["total_ms"] / steps
    peak, _ = peak_hbm()
    out = {"value": cells / (ms / 1e3) / 1e6, "unit": UNIT, "ms_per_step": ms, "steps": steps,
           "grid": [npx, npy, npz], "bytes_per_cell_step": bytes_per_cell,
           "hbm_frac": bytes_per_cell * cells / (ms / 1e3) / 1e9 / peak,
           "stage_kernel_ms": tm["stage_ms"] / max(1, tm["stage_launches"])}
    if fp64_ms_per_step:
        out["speedup_vs_fp64"] = fp64_ms_per_step / ms
    return out


def fp32_error_run(R, local, grid, steps, flags=(), seed=None):
    """FP32-bulk against FP64 after `steps` steps from the same initial state: per-field
    relative L2 / Linf error on the interior (computed on the device, r3d_gpu_compare: no host
    copy of either state), total mass and energy drift of both, and the step time of both (CUDA
    events).  Both states stay on the device together (504 x 504 x 2048: 63 + 32 GB)."""
    seed = SEED if seed is None else seed
    base = ["--npx", str(grid[0]), "--npy", str(grid[1]), "--npz", str(grid[2]), "--seed", str(seed),
            "--gpu", str(local)] + list(flags)
    out = {"grid": list(grid), "steps": steps, "seed": seed, "flags": list(flags)}
    p64 = R.parse(base + ["--precision", "fp64"])
    p32 = R.parse(base + ["--precision", "fp32bulk"])
    totals, times, setup_s = {}, {}, {}
    with R.GpuSim(p64) as s64, R.GpuSim(p32) as s32:
        for prec, sim in (("fp64", s64), ("fp32bulk", s32)):
            t0 = time.perf_counter()
            sim.setup()  # the same initial state for both forms, built on the device
            setup_s[prec] = time.perf_counter() - t0
            m0, e0 = sim.totals()
            _, tm = sim.run_timed(steps)
            m1, e1 = sim.totals()
            totals[prec] = {"mass_drift": (m1 - m0) / m0, "energy_drift": (e1 - e0) / e0}
            times[prec] = tm["total_ms"] / steps
        err = s32.compare(s64)
    out.update({"device_setup_s": setup_s, "error": err, "max_rel_l2": max(v["rel_l2"] for v in err.values()),
                "totals": totals, "ms_per_step": times, "speedup": times["fp64"] / times["fp32bulk"],
                "mcell_updates_per_s": {k: grid[0] * grid[1] * grid[2] / (v / 1e3) / 1e6 for k, v in times.items()}})
    return out


# The plume workload: FP32-bulk 504 x 504 x 2048 with the reference's plume top boundary
# (tp 2, itcon 1; src/bcon.cpp:43-70), seed 11, 50 steps, FP64 alongside
PLUME = ["--tp", "2", "--tc", "0", "--xp", "10", "--yp", "10", "--zp", "0", "--hh", "1"]


def adjoint_run(R, local, steps=200, every=20):
    """Time of the discrete adjoint on the MHD 64x64x128 case: record `steps` steps with a
    checkpoint every `every` (200 and 20 by default), then the checkpointed reverse sweep (seed:
    d(kinetic energy)/dX).
    CUDA events on the library's stream bracket each call (device time, host gaps included);
    the wall clock around the synchronous calls is reported beside them."""
    import numpy as np
    import torch

    p = R.parse(["--npx", "64", "--npy", "64", "--npz", "128", "--lmag", "1", "--beta", "10", "--rm", "1",
                 "--ampb", "0.1", "--bfh", "2", "--bzp", "20", "--seed", "5", "--gpu", str(local)])
    st = R.HostState.setup(p)
    with R.GpuSim(p) as sim:
        stream = torch.cuda.ExternalStream(sim.stream, device=torch.device("cuda", local))
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        sim.upload(st)
        sim.adjoint_record(20, 20)  # warm-up (allocates the workspace)
        fin = st.copy()
        sim.download(fin)
        seed = {n: np.zeros_like(a) for n, a in fin.fields.items()}
        sim.adjoint_backward(seed)  # warm-up of the reverse kernels
        sim.upload(st)
        torch.cuda.synchronize(local)
        t0 = time.perf_counter()
        ev[0].record(stream)
        sim.adjoint_record(steps, every)
        ev[1].record(stream)
        t1 = time.perf_counter()
        sim.download(fin)
        ro = fin.fields["ro"]
        for n in ("ru", "rv", "rw"):
            seed[n] = fin.fields[n] / ro
        seed["ro"] = -0.5 * (fin.fields["ru"] ** 2 + fin.fields["rv"] ** 2 + fin.fields["rw"] ** 2) / ro ** 2
        torch.cuda.synchronize(local)
        t2 = time.perf_counter()
        ev[2].record(stream)
        sim.adjoint_backward(seed)
        ev[3].record(stream)
        t3 = time.perf_counter()
        torch.cuda.synchronize(local)
        fwd_ms, bwd_ms = ev[0].elapsed_time(ev[1]), ev[2].elapsed_time(ev[3])
        mem = sim.adjoint_memory_bytes
    cells = 64 * 64 * 128
    return {"grid": [64, 64, 128], "steps": steps, "checkpoint_every": every,
            "forward_record_ms": fwd_ms, "backward_ms": bwd_ms, "backward_over_forward": bwd_ms / fwd_ms,
            "wall_ms": {"forward_record": (t1 - t0) * 1e3, "backward": (t3 - t2) * 1e3},
            "adjoint_mcell_steps_per_s": cells * steps / (bwd_ms / 1e3) / 1e6, "adjoint_device_bytes": mem,
            "note": "CUDA events on the library stream around each synchronous C ABI call (the "
                    "backward includes its seed upload and gradient download); wall_ms: host clock"}


def reference_layout(ncores: int):
    """Thread-ranks x OpenMP threads of the reference CPU run on ncores host threads (the
    reference needs npez >= 2 ranks)."""
    ranks = 2
    return ranks, max(1, ncores // ranks)


REF_BUDGET_S = 330.0  # wall time the reference arm's W + K steps may take (3 + 60 full steps: ~290 s)


def reference_depth(ranks: int, threads: int, steps: int) -> int:
    """Planes of the reference arm's grid: all of the benchmark grid's when W + K of its steps
    fit REF_BUDGET_S (R3D_REF_BUDGET_S overrides) on this host, else the depth that does (a
    bounded sample of the same planes; at least 32).  The step time is modelled as a + b *
    planes from one timed step on 32 and one on 64 planes of the grid."""
    from oracle import Reference

    budget = float(os.environ.get("R3D_REF_BUDGET_S", REF_BUDGET_S))
    if GRID[2] <= 32:
        return GRID[2]

    def one_step(depth):
        fl = ["--npx", str(GRID[0]), "--npy", str(GRID[1]), "--npz", str(depth), "--npey", "1"]
        return Reference.time_steps(fl, ranks, SEED, 0, 1, threads)[1]

    t32, t64 = one_step(32), one_step(64)
    b = max((t64 - t32) / 32, 1e-9)
    a = max(t32 - 32 * b, 0.0)
    if steps * (a + b * GRID[2]) <= budget:
        return GRID[2]
    return min(GRID[2], max(32, int((budget / steps - a) / b) // 8 * 8))


def run_reference_arm(args, world, rank, pg):
    """The reference's own CPU implementation (src/*.cpp compiled unmodified, thread-rank MPI
    stand-in, OpenMP): set-up, W untimed steps, K timed steps on the benchmark grid, or on a
    shallower grid of the same planes when W + K full steps would take more than a few minutes
    (reference_depth)."""
    if rank != 0:
        return 0
    base = {"metric": METRIC, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "impl": "reference"}
    try:
        from oracle import Reference

        if not Reference.available():
            emit({**base, "impl": "reference",
                  "unavailable": "reference CPU build oracle/_ref/libr3dref.so not present"})
            return 0
        ncores = os.cpu_count() or 1
        ranks, threads = reference_layout(ncores)
        depth = reference_depth(ranks, threads, args.warmup + args.steps)
        fl = ["--npx", str(GRID[0]), "--npy", str(GRID[1]), "--npz", str(depth), "--npey", "1"]
        cells = GRID[0] * GRID[1] * depth
        sc, sec = Reference.time_steps(fl, ranks, SEED, args.warmup, args.steps, threads)
        v = cells * args.steps / sec / 1e6
        what = ("the full benchmark grid" if depth == GRID[2] and world == 1 else
                f"a bounded sample of the {GRID[0]}x{GRID[1]}x{GRID[2] * world} workload: {depth} of its planes")
        sample = (f"reference CPU sources compiled unmodified (-O2 -ffp-contract=off -fopenmp), "
                  f"{ranks} thread-ranks x {threads} OpenMP threads on {ncores} host threads, grid "
                  f"{GRID[0]}x{GRID[1]}x{depth} ({what}), {args.warmup} untimed + "
                  f"{args.steps} timed RK3 steps, seed {SEED}")
        out = {**base, "value": v, "ms_per_step": sec / args.steps * 1e3, "scaling": "weak",
               "vs_baseline": None, "dtype": "f64", "data": "synthetic",
               "config": {"workload": f"FP64 hydro {GRID[0]}x{GRID[1]}x{GRID[2] * world} default physics seed {SEED}",
                          "grid": [GRID[0], GRID[1], GRID[2] * world], "sampled_grid": [GRID[0], GRID[1], depth]},
               "final_dt": sc["dt"],
               "cpu_baseline": {"value": v, "unit": UNIT, "cores": ranks * threads, "kind": "reference",
                                "sample": sample},
               "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        emit(out)
    except Exception as e:
        emit({**base, "unavailable": f"reference CPU run failed: {e}"})
    return 0


_RESULT = None  # stdout as it was at start: the JSON line goes there and nowhere else


def emit(obj):
    """Print the one JSON result line on the original stdout."""
    out = _RESULT if _RESULT is not None else sys.stdout
    out.write(json.dumps(obj) + "\n")
    out.flush()


def main():
    # The JSON line must be the only output on stdout.  Libraries print there too (NCCL writes
    # its version line at any NCCL_DEBUG level from WARN up, and INFO logs), so file descriptor 1
    # is pointed at stderr for the whole run and the result is written to a duplicate of the
    # original stdout.
    global _RESULT
    sys.stdout.flush()
    _RESULT = os.fdopen(os.dup(1), "w")
    os.dup2(2, 1)
    # NCCL's communicator lines (rank counts) go to stderr with the rest of the log
    os.environ.setdefault("NCCL_DEBUG", "INFO")
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extra", action="store_true", help="skip the FP32-bulk and MHD side measurements")
    ap.add_argument("--grid", type=int, nargs=3, metavar=("NPX", "NPY", "NPZ"),
                    help="another grid (small cases for profiling); the default is the benchmark grid")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32bulk"],
                    help="form of the headline run (fp64 is the benchmark; fp32bulk for profiling)")
    ap.add_argument("--slabs", action="store_true",
                    help="run a single GPU through the NCCL z-slab path (one rank), as N > 1 does")
    ap.add_argument("--mhd", action="store_true",
                    help="MHD (--lmag 1 --beta 10 --rm 1, layer ampb 0.1 bfh 2 bzp 20; for profiling cases)")
    ap.add_argument("--fp32-error", type=int, nargs=4, metavar=("NPX", "NPY", "NPZ", "STEPS"),
                    help="only measure FP32-bulk against FP64 on this grid after STEPS steps and print it")
    ap.add_argument("--plume", action="store_true",
                    help="with --fp32-error: plume forcing tp=2 tc=0 xp=yp=10 zp=0 hh=1, seed 11")
    ap.add_argument("--dry-launch", action="store_true",
                    help="start and join the ranks (gloo) and report them, without GPU work")
    ap.add_argument("--adjoint", type=int, nargs=2, metavar=("STEPS", "EVERY"),
                    help="only the adjoint leg (MHD 64x64x128), STEPS recorded with a checkpoint every EVERY")
    ap.add_argument("--reference-gpu-leg", action="store_true",
                    help="only the reference's own GPU driver on the benchmark grid (or --grid), printed as one line")
    args = ap.parse_args()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return spawn_ranks(args.gpus)
    if args.adjoint:
        import r3d_b200 as R

        emit(adjoint_run(R, 0, *args.adjoint))
        return 0
    if args.fp32_error:
        import r3d_b200 as R

        g = args.fp32_error
        emit(fp32_error_run(R, 0, g[:3], g[3], PLUME if args.plume else (), seed=11 if args.plume else None))
        return 0
    global GRID, FLAGS
    if args.grid:
        GRID = tuple(args.grid)
        FLAGS = ["--npx", str(GRID[0]), "--npy", str(GRID[1]), "--npz", str(GRID[2])]
    if args.reference_gpu_leg:
        emit(reference_gpu_leg())
        return 0
    if args.warmup < 3:
        args.warmup = 3
    world, rank, local, pg = dist_init()
    if world != args.gpus:
        print(f"bench: --gpus {args.gpus} but {world} ranks joined", file=sys.stderr)
        if pg is not None:
            pg.destroy_process_group()
        return 2
    if args.dry_launch:
        rc = dry_launch(args, world, rank, pg)
        if pg is not None:
            pg.destroy_process_group()
        return rc
    if args.impl == "reference":
        rc = run_reference_arm(args, world, rank, pg)
        if pg is not None:
            pg.destroy_process_group()
        return rc

    import numpy as np

    import r3d_b200 as R

    fp32 = args.precision == "fp32bulk"
    bytes_step = 200.0 if fp32 else BYTES_PER_CELL_STEP
    mag = (["--lmag", "1", "--beta", "10", "--rm", "1", "--ampb", "0.1", "--bfh", "2", "--bzp", "20"]
           if args.mhd else [])
    if args.mhd:
        bytes_step = 640.0
    if world == 1 and not args.slabs:
        p = R.parse(FLAGS + mag + ["--seed", str(SEED), "--gpu", str(local), "--precision", args.precision])
        cells = GRID[0] * GRID[1] * GRID[2]
        t_setup = time.perf_counter()
        st = R.HostState.setup(p)
        t_setup = time.perf_counter() - t_setup
        sim = R.GpuSim(p)
    else:
        # weak scaling: the domain is npx x npy x (npz * N), one z slab of npz planes per GPU,
        # ghost planes exchanged over NCCL after every stage, dt limits all-reduced per step
        from r3d_b200 import dist as D

        p = R.parse(["--npx", str(GRID[0]), "--npy", str(GRID[1]), "--npz", str(GRID[2] * world),
                     "--seed", str(SEED), "--gpu", str(local), "--precision", args.precision] + mag)
        z0, nz = D.slab_of(p.npz, rank, world)
        cells = GRID[0] * GRID[1] * nz
        t_setup = time.perf_counter()
        st = R.HostState.setup_slab(p, z0, nz)
        t_setup = time.perf_counter() - t_setup
        sim = R.GpuSim(p, slab=(z0, nz))
        sim.halo_init(D.share_unique_id(rank, pg), rank, world)
    t_upload = time.perf_counter()
    sim.upload(st)
    t_upload = time.perf_counter() - t_upload
    with ClockSampler(local) as clk:
        sim.run(args.warmup)                     # untimed warm-up
        clk.wait_first()
        barrier(pg)
        sc, tm = sim.run_timed(args.steps)       # synchronises on exit
    refolds = sim.debug_dt_filter()              # full dt re-evaluations since the upload
    barrier(pg)
    total_ms = allmax(pg, tm["total_ms"])
    stage_avg_ms = tm["stage_ms"] / max(1, tm["stage_launches"])
    ms_per_step = total_ms / args.steps
    value = world * cells * args.steps / (total_ms / 1e3) / 1e6

    # end to end through the C ABI with host buffers: upload from pinned host memory, K steps
    # that each return the scalars to the host (as step_gpu does), download of the state.
    import torch

    pinned = {}
    for n, a in st.fields.items():
        t = torch.empty(a.shape, dtype=torch.float64, pin_memory=torch.cuda.is_available())
        t.numpy()[...] = a
        pinned[n] = t
    st_pinned = R.HostState({n: t.numpy() for n, t in pinned.items()}, st.lines, dict(st.scalars))
    e2e_steps = args.steps
    barrier(pg)
    t0 = time.perf_counter()
    sim.upload(st_pinned)
    for _ in range(e2e_steps):
        sim.step()
    sim.download(st_pinned)
    e2e_s = allmax(pg, time.perf_counter() - t0)
    state_bytes = sum(a.nbytes for a in st.fields.values())
    e2e = {"value": world * cells * e2e_steps / e2e_s / 1e6, "unit": UNIT,
           "h2d_bytes_per_step": int(state_bytes / e2e_steps) + 64,
           "d2h_bytes_per_step": int(state_bytes / e2e_steps) + 64,
           "note": "host state uploaded once and downloaded once per K-step job through the C ABI "
                   "(gpu_upload/step_gpu/gpu_download pattern); bytes amortised per step, plus the "
                   "per-step scalar read-back"}

    peak, peak_kind = peak_hbm()
    alg_bytes_launch = cells * bytes_step / 3.0
    achieved = alg_bytes_launch / (stage_avg_ms / 1e3) / 1e9
    traffic = None if (fp32 or args.mhd) else stage_traffic_per_launch(cells)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic, "peak_source": f"{peak_kind} hbm_gbs",
                "kernel": ("stage_fp32" if fp32 else "stage_fp64") + " (fused FLUXES + RK3 stage update)",
                "step_frac": (cells * bytes_step / (ms_per_step / 1e3) / 1e9) / peak}

    # the same initial state built on the device (r3d_gpu_setup), for the set-up time
    t_dev = time.perf_counter()
    sim.setup()
    t_dev = time.perf_counter() - t_dev
    sim.close()
    extra = {"setup": {"host_setup_s": t_setup, "upload_s": t_upload, "device_setup_s": t_dev,
                       "note": "initial state of the headline grid: host set-up (arrays on the host) + "
                               "upload, against r3d_gpu_setup (no host 3D arrays); wall clock"}}
    if not args.no_extra and not args.grid and not fp32 and world == 1 and not args.slabs and not args.mhd:
        extra["fp32bulk_504x504x512"] = side_run(R, FLAGS + ["--seed", str(SEED), "--precision", "fp32bulk",
                                                             "--gpu", str(local)], args.steps, args.warmup,
                                                 200.0, ms_per_step)
        extra["mhd_fp64_126x126x256"] = side_run(R, ["--npx", "126", "--npy", "126", "--npz", "256", "--lmag", "1",
                                                     "--beta", "10", "--rm", "1", "--ampb", "0.1", "--bfh", "2",
                                                     "--bzp", "20", "--seed", "7", "--gpu", str(local)],
                                                 max(args.steps, 20), args.warmup, 640.0, None)
        extra["adjoint_mhd_64x64x128"] = adjoint_run(R, local)
        extra["fp32bulk_error_504x504x512_100steps"] = fp32_error_run(R, local, GRID, 100)
        extra["fp32bulk_plume_504x504x2048_50steps"] = fp32_error_run(R, local, (504, 504, 2048), 50,
                                                                              PLUME, seed=11)
        extra["reference_gpu_driver_504x504x512"] = reference_gpu_run(ms_per_step)
    cpu = None
    if rank == 0 and not args.no_cpu_baseline and world == 1:
        cpu = cpu_reference_sample()
    if rank == 0:
        out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64" if fp32 else "f64",
               "data": "synthetic",
               "config": {"workload": f"{'FP32-bulk' if fp32 else 'FP64'} {'MHD' if args.mhd else 'hydro'} {GRID[0]}x{GRID[1]}x{GRID[2]}, default physics, "
                                      f"polytrope + RAN2 seed {SEED} ampt 0.005",
                          "grid": list(GRID), "precision": args.precision, "bit_exact": not fp32,
                          "l2": "inputs 16 GB >> 126 MB L2 (no flush needed)",
                          "parallelism": ("1 GPU" if world == 1 and not args.slabs else
                                          f"{world} z-slabs of {GRID[0]}x{GRID[1]}x{GRID[2]}, one per GPU "
                                          f"(NCCL ghost planes per stage, dt all-reduce per step)")},
               "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
               "gpu_launches": int(tm["total_launches"]), "clocks": clk.summary(),
               "final_dt": sc["dt"],
               "dt_refolds": {"count": refolds, "steps": args.warmup + args.steps,
                              "note": "full re-evaluations of the third stage's filtered dt limits"},
               "extra": extra}
        emit(out)
    if pg is not None:
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
