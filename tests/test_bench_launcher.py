"""The multi-GPU launcher of bench.py on CPU: --gpus 2 starts two ranks
(torch.distributed.run, gloo without CUDA), every rank takes its
work-balanced shard of the global batch, and rank 0 prints one line with
n_gpus = 2 whose shards cover the whole batch."""
import json
import subprocess
import sys
from pathlib import Path

REPO = Path(__file__).resolve().parent.parent


def test_bench_spawns_ranks_and_shards():
    out = subprocess.run(
        [sys.executable, str(REPO / "bench.py"), "--gpus", "2", "--dry-run",
         "--tracks", "20000"],
        capture_output=True, text=True, timeout=300, check=True)
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out.stdout + out.stderr
    line = json.loads(lines[0])
    assert line["n_gpus"] == 2
    assert line["global_batch"] == 40000
    assert line["rank0_range"][0] == 0
    assert 0 < line["largest_shard"] < 40000


def test_bench_rejects_gpus_other_than_world_size(monkeypatch):
    monkeypatch.setenv("WORLD_SIZE", "3")
    out = subprocess.run(
        [sys.executable, str(REPO / "bench.py"), "--gpus", "2", "--dry-run"],
        capture_output=True, text=True, timeout=120)
    assert out.returncode != 0
    assert "WORLD_SIZE" in out.stderr
