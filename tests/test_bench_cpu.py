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


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        q.put((rank, bench.max_over_ranks(1.5 + rank, dist, device="cpu")))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    """bench.py's multi-GPU time is the slowest rank's: two gloo ranks on CPU."""
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = dict(q.get(timeout=10) for _ in range(2))
    assert got == {0: 2.5, 1: 2.5}


def test_max_over_ranks_single_process():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.max_over_ranks(3.25, None) == 3.25


@pytest.mark.skipif(not (ROOT / "epigpu_b200" / "bin" / "epiGPU").exists() or
                    not (ROOT / "oracle" / "_ref" / "plinkref").exists(),
                    reason="host program or the reference's data-mode oracle not built")
@pytest.mark.parametrize("impl", ["ours", "reference"])
def test_datamode_workload(impl):
    """The data-mode measurement (PLINK text -> .epigpu on the host): one JSON line per arm, and
    the two arms' .epigpu files byte-identical."""
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--workload", "datamode", "--impl", impl,
                        "--steps", "1", "--warmup", "0"], capture_output=True, text=True, timeout=300, cwd=str(ROOT))
    assert r.returncode == 0, r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["unit"] == "MB/s" and d["value"] > 0 and d["config"]["identical_to_other_arm"] is True
    assert (d.get("impl") == "reference") == (impl == "reference")
