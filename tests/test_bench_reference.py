"""The benchmark's reference arm on the host: `bench.py --impl reference` times the reference's own
CPU cascade (the reference build in oracle/_ref) and prints one JSON line with the benchmark's
metric, its CPU baseline and an end-to-end object without host-device copies; under a multi-rank
launch only rank 0 runs and prints."""
import json
import os
import subprocess
import sys

import pytest

from oracle import ref

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(env_extra):
    env = dict(os.environ, **env_extra)
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1", "--warmup", "1"],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    return [json.loads(l) for l in p.stdout.splitlines() if l.startswith("{")]


@pytest.mark.skipif(not ref.available(), reason="reference build oracle/_ref/libccnn_ref.so not present")
def test_reference_arm_line():
    lines = _run({"WORLD_SIZE": "1", "RANK": "0"})
    assert len(lines) == 1
    d = lines[0]
    assert d["impl"] == "reference" and d["unit"] == "frames/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] == 1 and d["n_gpus"] == 1
    assert "1920x1080" in d["config"]["workload"]
    assert d["e2e"] == {"value": d["value"], "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]


def test_reference_arm_other_ranks_print_nothing():
    assert _run({"WORLD_SIZE": "2", "RANK": "1"}) == []
