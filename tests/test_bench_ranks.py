"""The multi-process path of bench.py on CPU: two gloo ranks reduce their
per-rank times to the maximum (what `bench.py --gpus 2` reports), and a rank
with one process returns its own values."""
import os
import socket
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        got = bench.max_over_ranks([10.0 + rank, 5.0 - rank, 7.0], dist, "cpu")
        out[rank] = got
    finally:
        dist.destroy_process_group()


def test_max_over_two_gloo_ranks():
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_rank, args=(2, _free_port(), out), nprocs=2, join=True)
    assert out[0] == out[1] == [11.0, 5.0, 7.0]


def test_single_process_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks([1, 2.5], None, "cpu") == [1.0, 2.5]


def _run_bench(args, env_extra=None):
    import json
    import subprocess
    env = dict(os.environ, **(env_extra or {}))
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py")] + args, cwd=ROOT, env=env,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]
    return lines


def test_reference_arm_line_contract():
    """`bench.py --impl reference` times the CPU restatement on the host cores
    and prints the same metric, unit and config as the GPU arm, with the
    reference-arm keys (impl, cpu_baseline, e2e with no host<->device bytes)."""
    args = ["--impl", "reference", "--steps", "2", "--warmup", "1", "--instances", "2", "--log-n", "8",
            "--queries", "8"]
    (line,) = _run_bench(args)
    assert line["impl"] == "reference" and line["unit"] == "ms" and line["higher_is_better"] is False
    assert line["value"] > 0 and line["value"] == line["ms_per_step"] == line["e2e"]["value"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    base = line["cpu_baseline"]
    # each step proves the whole workload (no sample scaled up)
    assert base["kind"] == "port" and base["cores"] >= 1 and "whole workload (2 instances" in base["sample"]
    assert len(base["steps_ms"]) == 2 and line["value"] == base["value"]
    assert line["config"]["instances"] == 2 and line["config"]["log_rows"] == 8
    # under torchrun only rank 0 runs and prints; the other ranks exit 0 without work
    assert _run_bench(args, {"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"}) == []


def test_device_idle_accounting():
    """Gaps between recorded launches count in the phase of the launch that
    ends them; overlapping launches leave no gap."""
    sys.path.insert(0, ROOT)
    import bench
    timeline = [("k_a", 0, 0.0, 1.0), ("k_b", 0, 0.5, 1.0), ("k_c", 1, 2.0, 0.5), ("k_d", 2, 3.0, 1.0),
                ("k_e", 5, 4.25, 0.25)]
    got = bench.device_idle(timeline, ["round 0", "round 2", "deep"])
    assert got == {"total": 1.25, "span": 4.5, "by_phase": {"round 2": 0.5, "deep": 0.5, "after last phase": 0.25}}
    assert bench.device_idle([], ["round 0"]) is None
