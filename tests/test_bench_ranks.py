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
