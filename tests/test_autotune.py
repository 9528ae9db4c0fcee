"""Autotuner logic on a fake context (no GPU): coordinate descent keeps the
fastest value of each parameter, and results round-trip through the cache."""
import json

import pytest

from loom_b200 import autotune as AT


class FakeContext:
    """Commit time is a fixed function of the tuning values; minimum at
    p2_leaf_min_per_sm=64, merkle_tail=128, everything else at its default."""
    DEFAULTS = {"p2_leaf_min_per_sm": 128, "p2_node_min_per_sm": 512, "p2_inject_min_per_sm": 128,
                "merkle_tail": 32, "merkle_subtree": 16, "inject_block": 32, "leaf_block": 128, "lde_split": 1,
                "lde_fwd_threads": 512}

    def __init__(self):
        self.t = dict(self.DEFAULTS)
        self.prof = False

    def device_key(self):
        return "fake-gpu|sm148|build"

    def set_leaf_mapping(self, m):
        pass

    def tuning(self):
        return dict(self.t)

    def set_tuning(self, n, v):
        assert n in self.t
        self.t[n] = v

    def apply_tuning(self, params):
        self.t.update(params)

    def commit_root(self, groups):
        return None

    def profile(self, on):
        self.prof = on

    def profile_report(self):
        cost = 1.0 + abs(self.t["p2_leaf_min_per_sm"] - 64) / 100 + abs(self.t["merkle_tail"] - 128) / 100
        cost += 0.5 * (self.t["inject_block"] != 32) + 0.5 * (self.t["leaf_block"] != 128)
        # the NTT: the split LDE with 1024-thread coset blocks is fastest here
        lde = 1.0 if self.t["lde_split"] == 0 else 0.6 + 0.1 * (self.t["lde_fwd_threads"] != 1024)
        return {"hash_leaves": {"ms": cost, "launches": 1, "bytes": 0, "perms": 0},
                "lde": {"ms": lde, "launches": 1, "bytes": 0, "perms": 0}}


def test_coordinate_descent_and_cache(tmp_path, monkeypatch):
    monkeypatch.setenv("LOOM_B200_TUNING", str(tmp_path / "t.json"))
    monkeypatch.setattr(AT, "SHAPES", ((1, 4, 1),))
    ctx = FakeContext()
    res = AT.autotune(ctx, runs=1)
    assert res["source"] == "measured"
    assert res["params"]["p2_leaf_min_per_sm"] == 64 and res["params"]["merkle_tail"] == 128
    assert res["params"]["inject_block"] == 32 and res["params"]["leaf_block"] == 128
    assert res["params"]["lde_split"] == 1 and res["params"]["lde_fwd_threads"] == 1024
    assert res["ms_tuned"] < res["ms_default"]
    saved = json.load(open(tmp_path / "t.json"))
    assert saved["fake-gpu|sm148|build"]["params"] == res["params"]
    fresh = FakeContext()
    again = AT.autotune(fresh)
    assert again["source"] == "cache" and fresh.t == res["params"]


def test_candidates_are_valid_library_values():
    for name, values in AT.CANDIDATES.items():
        for v in values:
            if name in ("merkle_tail", "inject_block", "leaf_block"):
                assert v & (v - 1) == 0
            if name == "merkle_tail":
                assert 2 <= v <= 1024
            if name == "merkle_subtree":
                assert v == 0 or (2 <= v <= 1024 and v & (v - 1) == 0)
            if name in ("inject_block", "leaf_block"):
                assert 32 <= v <= 1024
            if name == "lde_split":
                assert v in (0, 1)
            if name == "lde_fwd_threads":
                assert v in (256, 512, 1024)
