"""Autotuner for the launch-shape choices of libloom_gpu (lg_ctx_set_tuning in
include/loom_gpu.h): the Poseidon2 lane mapping thresholds (leaves, injection
chains, Merkle levels), the width below which Merkle levels run in one block,
block sizes, and the NTT's launch structure (the LDE fused into one block per
lane or split into an inverse launch and one block per coset, and the coset
blocks' thread count).  Proof bytes never depend on them; only time does.

For each parameter in turn (coordinate descent from the current values), every
candidate value is timed on representative commits: the round commit of many
equal modules (LDE, leaf hashing plus a long injection chain per node), one
wide column batch, and small trees whose top levels are latency bound.  Times
are the library's CUDA events around its LDE and Poseidon2 kernels (median of
a few runs), summed over the shapes.  The winner of every parameter
is kept, and the result is cached per GPU (name, SM count) and library build
in a JSON file: $LOOM_B200_TUNING, else ~/.cache/loom_b200/tuning.json.
"""
from __future__ import annotations

import hashlib
import json
import os
import statistics
import time
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import _lib
from . import field as F

CANDIDATES: Dict[str, Sequence[int]] = {
    "lde_split": (0, 1),
    "lde_fwd_threads": (256, 512, 1024),
    "p2_leaf_min_per_sm": (32, 64, 128, 256, 512),
    "p2_inject_min_per_sm": (64, 128, 256, 512, 1 << 20),
    "p2_node_min_per_sm": (128, 256, 512, 1024, 2048),
    "merkle_tail": (16, 32, 64, 128),
    "merkle_subtree": (0, 8, 16, 32, 64),
    "inject_block": (32, 64, 128),
    "leaf_block": (64, 128, 256),
}
TIMED_KERNELS = ("lde", "lde_inv", "hash_leaves", "merkle_level", "merkle_inject", "merkle_tail")
# (groups, log2 rows per group, base columns per group): the round commit of
# 40 plonk modules of 2^14 rows, a wide batch, a mid-size batch, small trees
SHAPES: Tuple[Tuple[int, int, int], ...] = ((40, 14, 3), (1, 16, 16), (8, 12, 3), (4, 9, 4))


def cache_path() -> str:
    return os.environ.get("LOOM_B200_TUNING") or os.path.join(os.path.expanduser("~"), ".cache", "loom_b200",
                                                              "tuning.json")


def _device_key(ctx) -> str:
    if hasattr(ctx, "device_key"):
        return ctx.device_key()
    import torch
    props = torch.cuda.get_device_properties(ctx.device)
    with open(_lib.LIB_PATH, "rb") as f:
        build = hashlib.sha1(f.read()).hexdigest()[:16]
    return f"{props.name}|sm{props.multi_processor_count}|{build}"


def _load_cache() -> dict:
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def cached(ctx) -> Optional[Dict[str, int]]:
    """Tuned values for this GPU and library build, if the cache holds them."""
    entry = _load_cache().get(_device_key(ctx))
    return dict(entry["params"]) if entry else None


def _shape_groups(seed: int) -> List[List[dict]]:
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for groups, logn, cols in SHAPES:
        gs = []
        for _ in range(groups):
            base = [F.to_mont(rng.integers(0, F.P, 1 << logn, dtype=np.uint64).astype(np.uint32)) for _ in range(cols)]
            gs.append({"rows": 1 << logn, "base": base})
        out.append(gs)
    return out


def _time_shapes(ctx, shapes: List[List[dict]], runs: int) -> float:
    total = 0.0
    for gs in shapes:
        ctx.commit_root(gs)  # warm (tables, pools)
        samples = []
        for _ in range(runs):
            ctx.profile(True)
            ctx.commit_root(gs)
            rep = ctx.profile_report()
            ctx.profile(False)
            samples.append(sum(rep[k]["ms"] for k in TIMED_KERNELS if k in rep))
        total += statistics.median(samples)
    return total


def autotune(ctx, force: bool = False, runs: int = 3, save: bool = True, log=None) -> dict:
    """Tunes `ctx` (a loom_b200.Context) and returns {"params", "source",
    "seconds", "ms_default", "ms_tuned"}.  A cached result for this GPU and
    build is applied without measuring unless `force`."""
    t0 = time.time()
    if not force:
        params = cached(ctx)
        if params is not None:
            ctx.apply_tuning(params)
            return {"params": params, "source": "cache", "seconds": round(time.time() - t0, 3)}
    ctx.set_leaf_mapping(0)
    shapes = _shape_groups(0x70E)
    best = ctx.tuning()
    best_ms = ms_default = _time_shapes(ctx, shapes, runs)
    for name, values in CANDIDATES.items():
        keep = best[name]
        for v in values:
            if v == keep:
                continue
            ctx.set_tuning(name, v)
            ms = _time_shapes(ctx, shapes, runs)
            if log:
                log(f"autotune {name}={v}: {ms:.3f} ms (best {best_ms:.3f} at {best[name]})")
            if ms < best_ms * 0.99:  # a change must win by more than the noise
                best_ms, best[name] = ms, v
        ctx.set_tuning(name, best[name])
    res = {"params": best, "source": "measured", "seconds": round(time.time() - t0, 3),
           "ms_default": round(ms_default, 4), "ms_tuned": round(best_ms, 4)}
    if save:
        data = _load_cache()
        data[_device_key(ctx)] = {"params": best, "ms_default": res["ms_default"], "ms_tuned": res["ms_tuned"],
                                  "when": time.strftime("%Y-%m-%dT%H:%M:%S")}
        try:
            os.makedirs(os.path.dirname(cache_path()), exist_ok=True)
            with open(cache_path(), "w") as f:
                json.dump(data, f, indent=1, sort_keys=True)
        except OSError as e:  # an unwritable cache costs a re-measurement next time, nothing else
            res["cache_error"] = str(e)
    return res
