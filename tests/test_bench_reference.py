"""bench.py's reference arm on the CPU: the reference's own CPU build
(oracle/_ref) timed on a bounded sample, printed as one JSON line with the
keys the benchmark contract asks for."""
import json
import os
import subprocess
import sys

import pytest

from oracle import refjob

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(not refjob.available("langte"), reason="reference build missing")
def test_reference_arm_prints_one_contract_line():
    # a 16^3 box here (the arm's default is the benchmark's 128^3)
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--size", "16",
                          "--steps", "1", "--warmup", "1"], cwd=ROOT, capture_output=True,
                         text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["steps"] == 1 and d["warmup"] == 1
    assert d["unit"] == "atom-steps/s" and d["value"] > 0 and d["higher_is_better"] is True
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
    assert "workload" in d["config"]


@pytest.mark.skipif(not refjob.available("langte"), reason="reference build missing")
def test_reference_arm_under_torchrun_prints_from_rank_zero_only():
    # launched as the multi-GPU benchmark is: rank 0 runs and prints, the
    # other ranks exit 0 without work
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    out = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
                          "--nproc-per-node", "2", "--master-addr", "127.0.0.1",
                          "--master-port", str(port), "bench.py", "--impl", "reference",
                          "--size", "16", "--gpus", "2", "--steps", "1", "--warmup", "1"],
                         cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
