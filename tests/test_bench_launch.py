"""bench.py's launch contract on the CPU: `--gpus N` outside a launcher starts N ranks itself
(torch.distributed.run on 127.0.0.1), a launcher whose WORLD_SIZE differs from --gpus is
refused before any work, and the reference arm under two ranks prints exactly one JSON line
(rank 0 times the reference core on the host; the other rank exits without work)."""
import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _env(**extra):
    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK")}
    env.update(extra)
    return env


def test_world_size_mismatch_is_refused():
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--gpus", "2", "--impl", "reference"],
                       env=_env(WORLD_SIZE="3", RANK="0"), capture_output=True, text=True, timeout=300)
    assert r.returncode != 0
    assert "--gpus 2 but the launcher started WORLD_SIZE=3 ranks" in r.stderr
    assert r.stdout.strip() == ""


def test_reference_arm_under_two_ranks_prints_one_line(ref):
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--gpus", "2", "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], env=_env(), capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1, r.stdout
    line = lines[0]
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["unit"] == "Mpx/s"
    assert line["value"] > 0 and line["e2e"]["value"] == line["value"]
    assert line["cpu_baseline"]["kind"] == "reference" and line["e2e"]["h2d_bytes_per_step"] == 0
