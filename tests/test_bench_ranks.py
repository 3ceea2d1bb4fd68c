"""bench.py's rank plumbing on the host: `--gpus 2` without a launcher starts two ranks (gloo
here, NCCL on GPUs), times a step as the max over ranks, and only rank 0 prints, with
n_gpus == 2 — never one silent rank for two."""
from __future__ import annotations

import json
import os
import subprocess
import sys

from conftest import REPO


def test_gpus_two_runs_two_ranks_and_reports_them():
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="", MASTER_ADDR="127.0.0.1")
    env.pop("WORLD_SIZE", None)
    r = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--gpus", "2", "--dry-run", "--steps", "3",
                        "--warmup", "1"], capture_output=True, text=True, timeout=300, env=env, cwd=REPO)
    assert r.returncode == 0, r.stderr[-3000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["n_gpus"] == 2 and d["ranks"] == 2 and d["backend"] == "gloo"


def test_launcher_world_disagreeing_with_gpus_is_an_error():
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="", WORLD_SIZE="2", RANK="0", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--gpus", "4", "--dry-run"],
                       capture_output=True, text=True, timeout=120, env=env, cwd=REPO)
    assert r.returncode != 0 and "launcher started 2 ranks" in (r.stderr + r.stdout)
