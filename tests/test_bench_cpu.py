"""bench.py's reference arm on the host cores (no GPU): the JSON line the driver reads, and
the multi-rank rule (only rank 0 runs and prints)."""
import json
import os
import subprocess
import sys

import pytest

import oracles

ROOT = __import__("pathlib").Path(__file__).resolve().parents[1]

needs_ref = pytest.mark.skipif(not oracles.have_ref(), reason="reference kernels (oracle/_ref) not built")


def _run(env_extra, *args):
    env = dict(os.environ, **env_extra)
    return subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", *args],
                          capture_output=True, text=True, timeout=300, env=env, cwd=str(ROOT))


@needs_ref
def test_reference_arm_prints_one_json_line():
    r = _run({}, "--workload", "cfg1", "--steps", "1", "--warmup", "1")
    assert r.returncode == 0, r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "pairs/s" and d["value"] > 0
    assert d["higher_is_better"] is True and d["steps"] == 1 and d["warmup"] == 1
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["config"]["workload"].startswith("cfg1")


def test_reference_arm_other_ranks_print_nothing():
    r = _run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"}, "--workload", "cfg1", "--steps", "1",
             "--warmup", "1")
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
