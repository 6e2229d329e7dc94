"""bench.py's reference arm on the CPU: the reference engine compiled from its
own source (oracle/_ref) timed on the plain workload, one JSON line in the
bench contract's form."""
import json
import os
import subprocess
import sys

import pytest

from conftest import REPO

LIB = os.path.join(REPO, "oracle", "_ref", "libref_accelerate.so")


@pytest.mark.skipif(not os.path.exists(LIB), reason="reference engine not built (oracle/build_oracle.py)")
def test_reference_arm_json_line():
    out = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "1", "--cpu-procs", "2"], cwd=REPO, capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == "swap_evals_per_sec" and d["unit"] == "swap-evals/s"
    assert d["higher_is_better"] is True and d["n_gpus"] == 1 and d["steps"] == 1 and d["warmup"] == 1
    assert d["value"] > 0 and d["cpu_baseline"]["value"] == d["value"]
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] == 2
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["config"]["workload"].startswith("plain_gpu")


@pytest.mark.skipif(not os.path.exists(LIB), reason="reference engine not built (oracle/build_oracle.py)")
def test_reference_arm_under_torchrun_prints_once():
    """Launched like the multi-GPU bench (two ranks): rank 0 prints the line, the other rank exits 0."""
    out = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
                          "--master-addr", "127.0.0.1", "--master-port", "29533", os.path.join(REPO, "bench.py"),
                          "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "1", "--cpu-procs", "2"],
                         cwd=REPO, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
