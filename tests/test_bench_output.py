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
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1"],
                       cwd=ROOT, capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1, r.stdout
    out = json.loads(lines[0])
    assert out["impl"] == "reference" and out["value"] > 0
    assert out["cpu_baseline"]["kind"] == "reference" and out["cpu_baseline"]["cores"] >= 1
    assert out["e2e"]["h2d_bytes_per_step"] == 0
