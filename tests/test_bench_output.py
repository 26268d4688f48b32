"""bench.py's output contract: exactly one JSON line on stdout, whatever the libraries print.

Runs the CPU reference arm (the compiled reference sources on the host cores, one short step),
which needs no GPU; the GPU arm writes its line through the same function.
"""
import json
import os
import subprocess
import sys

import pytest

from conftest import ROOT


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libr3dref.so")),
                    reason="reference CPU build not present")
def test_reference_arm_prints_one_json_line():
    env = dict(os.environ, NCCL_DEBUG="INFO")  # a chatty library setting must not leak to stdout
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--grid", "48", "32", "16"],
                       cwd=ROOT, capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1, r.stdout
    out = json.loads(lines[0])
    assert out["impl"] == "reference" and out["value"] > 0
    assert out["cpu_baseline"]["kind"] == "reference" and out["cpu_baseline"]["cores"] >= 1
    assert out["e2e"]["h2d_bytes_per_step"] == 0
    assert out["config"]["grid"] == [48, 32, 16] and out["steps"] == 1 and out["warmup"] == 3
    assert out["config"]["sampled_grid"] == [48, 32, 16] and "full benchmark grid" in out["cpu_baseline"]["sample"]


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libr3dref.so")),
                    reason="reference CPU build not present")
def test_reference_arm_samples_planes_when_the_run_would_be_long():
    """W + K full-grid reference steps that would exceed the arm's time budget run on fewer of
    the grid's planes (at least 32), and the line says so."""
    env = dict(os.environ, R3D_REF_BUDGET_S="0.001")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--grid", "48", "32", "64"],
                       cwd=ROOT, capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    out = json.loads([ln for ln in r.stdout.splitlines() if ln.strip()][0])
    assert out["config"]["grid"] == [48, 32, 64] and out["config"]["sampled_grid"] == [48, 32, 32]
    assert "bounded sample" in out["cpu_baseline"]["sample"] and out["value"] > 0


@pytest.mark.parametrize("n", [2, 3])
def test_gpus_n_starts_and_joins_n_ranks(n):
    """`bench.py --gpus N` with no launcher starts the N ranks itself (one process per GPU,
    LOCAL_RANK = rank) and they join one group; --dry-launch stops before any GPU work, so this
    runs on the CPU.  Each rank reports its z slab of the weak-scaling domain and receives the
    transport id from rank 0."""
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", str(n), "--dry-launch"],
                       cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1, r.stdout
    out = json.loads(lines[0])
    assert out["n_gpus"] == n and out["requested"] == n
    assert [j["rank"] for j in out["joined"]] == list(range(n))
    assert [j["local_rank"] for j in out["joined"]] == list(range(n))
    assert all(j["uid_ok"] for j in out["joined"])
    assert sum(j["slab"][1] for j in out["joined"]) == out["domain"][2] == 512 * n


def test_gpus_n_under_a_launcher_with_the_wrong_world_fails():
    """Under a launcher (WORLD_SIZE set) a --gpus N that does not match the ranks that joined is
    refused loudly."""
    env = dict(os.environ, WORLD_SIZE="1", RANK="0", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2", "--dry-launch"],
                       cwd=ROOT, capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode != 0 and "2 but 1 ranks joined" in r.stderr
