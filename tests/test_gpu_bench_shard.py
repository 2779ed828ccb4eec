"""bench.py --shard on one GPU: the block-sharded config 3 solve on a single rank (the sharded
handle with no peers) prints its JSON line with strong scaling and a finite rate."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_bench_shard_one_rank():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--shard", "--steps", "3", "--warmup", "3"],
                         capture_output=True, text=True, timeout=900, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-3000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["scaling"] == "strong" and line["n_gpus"] == 1 and line["value"] > 0
    assert line["config"]["blocks"] == 24 and line["config"]["blocks_on_rank0"] == 24
    assert all(v == v for v in line["residual_rms"])
    assert line["gpu_launches"] > 0 and line["e2e"]["value"] > 0
