"""bench.py's multi-rank launch, on the CPU.

`bench.py --gpus N` without a torchrun environment starts N ranks itself
(torch.distributed.run on 127.0.0.1). The reference arm needs no GPU, so it
exercises that path here over gloo: both ranks must start, rank 0 alone prints
the one JSON line, and the line carries the GPU arm's config keys.
"""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_starts_every_rank_over_gloo():
    env = dict(os.environ)
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT"):
        env.pop(k, None)
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                          "--n", "16", "--steps", "2", "--warmup", "1"],
                         cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out.stdout
    line = json.loads(lines[0])
    assert line["impl"] == "reference"
    assert line["n_gpus"] == 2 and line["ranks_started"] == [0, 1]
    assert line["steps"] == 2 and line["warmup"] == 1
    for key in ("workload", "cells", "parallelism", "l2", "pcg_iterations_per_step", "pressure_ms_per_step"):
        assert key in line["config"], key
    assert line["config"]["cells"] == 16 ** 3 and line["config"]["pcg_iterations_per_step"] > 0
    assert line["cpu_baseline"]["kind"] == "port" and line["e2e"]["h2d_bytes_per_step"] == 0
