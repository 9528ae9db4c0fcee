"""Prove benchmark: loom's Poseidon2 prove phase on synthetic plonk-like
instances (default 40 modules x 2^14 rows, 200 FRI queries).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One JSON line on rank 0.  `value` = device-timed milliseconds per prove with
the witness resident in HBM (CUDA events on the library's stream, L2 flushed
between steps, max over ranks); `e2e` = the same call with the witness in
pinned host memory and the proof bytes returned to the host.  With N GPUs
every rank proves its own copy of the workload (replicas; the prove has no
cross-device exchange at this size).  `--impl reference` times the CPU
restatement of the reference prover (the reference is Go, which this
machine cannot build or run) on the host cores, one whole prove of the
same workload per step.
"""
from __future__ import annotations

import argparse
import gc
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "prove ms @40×2^14 plonk/Poseidon2, batched vs plain on 1 B200; serve p99 ms"
SLOW_REASONS = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--instances", type=int, default=40)
    ap.add_argument("--log-n", type=int, default=14)
    ap.add_argument("--queries", type=int, default=200)
    ap.add_argument("--cpu-steps", type=int, default=3, help="timed oracle proves of the CPU baseline (median)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--sweep", action="store_true",
                    help="kernel roofline sweep (LDE, Merkle commit, FRI fold, DEEP) instead of the prove bench")
    ap.add_argument("--sweep-only", type=str, default="",
                    help="comma-separated sweep items to run: lde, commit, fold, deep, or one size as kind:log2 "
                         "(lde:20 = the LDE of 2^20 output rows)")
    ap.add_argument("--serve-requests", type=int, default=2000, help="requests in the serving measurement (0 = skip)")
    ap.add_argument("--serve-shapes", type=int, default=8, help="distinct request shapes, replayed in turn")
    ap.add_argument("--serve-rate", type=str, default="32,64", help="Poisson arrival rates (requests/s) to sweep")
    ap.add_argument("--serve-streams", type=int, default=4)
    ap.add_argument("--no-c4", action="store_true",
                    help="skip the mixed-size lookup workload (40 modules, log2 rows 10-20, range lookup)")
    ap.add_argument("--no-tune", action="store_true", help="skip the autotuner (library defaults)")
    ap.add_argument("--retune", action="store_true", help="re-measure even if the tuning cache has this GPU")
    ap.add_argument("--streams", type=str, default="2,4,8,16",
                    help="concurrent proof streams for the throughput measurement")
    return ap.parse_args()


def workload_name(a):
    return f"{a.instances} plonk-like modules x 2^{a.log_n} rows (copy constraint, grand product), Poseidon2, {a.queries} queries"


# ---------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------- CPU baseline
def merge_lde(rep):
    """The LDE runs as an inverse launch ("lde_inv": read N, write coset 0)
    and a coset launch ("lde": write the other three cosets) when split; one
    LDE of a size class is the pair, 20 N bytes per lane in all."""
    inv = rep.pop("lde_inv", None)
    if inv is None:
        return
    l = rep.setdefault("lde", {"launches": inv["launches"], "ms": 0.0, "bytes": 0.0, "perms": 0.0})
    l["ms"] += inv["ms"]
    l["bytes"] += inv["bytes"]


def cpu_baseline(a, steps=1, warmup=0):
    """CPU restatement of the reference prover (oracle/: OpenMP over modules,
    columns, leaves and tree nodes, all host threads) proving the whole
    workload — every instance, the same program, witness and queries as the
    GPU arm; `warmup` untimed proves first, then the median of `steps`."""
    import oracle
    from loom_b200 import field as F, plonk
    oracle.lib()
    comp, wit = plonk.build(a.instances, 1 << a.log_n, seed=0x10AD)
    mont = [F.to_mont(w) for w in wit]
    for _ in range(warmup):
        oracle.prove(comp.words, mont, a.queries)
    times = []
    for _ in range(steps):
        t = time.perf_counter()
        oracle.prove(comp.words, mont, a.queries)
        times.append((time.perf_counter() - t) * 1e3)
    ms = statistics.median(times)
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return {"value": round(ms, 3), "unit": "ms", "cores": cores, "kind": "port",
            "sample": f"the whole workload ({a.instances} instances x 2^{a.log_n} rows, {a.queries} queries), "
                      f"median of {steps} proves after {warmup} untimed",
            "steps_ms": [round(t, 1) for t in times],
            "published_reference_ms": 4390.0,
            "published_reference_note": "the Go reference's own 4.39 s prove wall for 40 PLONK instances, "
                                        "Poseidon2, 200 queries on a 14-core Apple M4 (README.md:25); "
                                        "other hardware and an older build"}


def reference_arm(a, rank):
    if rank != 0:
        return
    # every timed step is one whole prove of the workload; the oracle keeps no
    # state between proves beyond its loaded library and touched pages, so one
    # untimed prove warms it whatever --warmup says
    base = cpu_baseline(a, steps=max(1, a.steps), warmup=min(a.warmup, 1))
    line = {"metric": METRIC, "value": base["value"], "unit": "ms", "n_gpus": a.gpus, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": base["value"], "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": {"workload": workload_name(a), "instances": a.instances, "log_rows": a.log_n,
                       "queries": a.queries},
            "impl": "reference", "cpu_baseline": base,
            "e2e": {"value": base["value"], "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the reference is Go and no Go toolchain exists here; this times the C++ restatement "
                    "of its prove path (oracle/) on all host threads, one whole prove per step, untimed "
                    "warm-up: one prove"}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------- kernel sweep
def sweep(a):
    """Kernel roofline sweep on seeded uniform data resident in HBM: batched
    coset LDE (2^16..2^24 output rows), Poseidon2 Merkle commit over LDEs,
    FRI fold of E6 vectors (2^18..2^24), DEEP over 256 columns at one point.
    One JSON line per measurement; per-kernel times are CUDA events on the
    library's stream."""
    import ctypes
    import faulthandler
    import torch
    from loom_b200 import Context, _lib
    faulthandler.enable()
    L = _lib.load()
    dev = torch.device("cuda:0")
    ctx = Context(0)
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except OSError:
        pass
    hbm = peaks.get("hbm_gbs", 6650.0)
    g = torch.Generator(device=dev)
    g.manual_seed(0x5EED)

    def field(n):
        return torch.randint(0, 0x7F000001, (n,), dtype=torch.int64, device=dev, generator=g).to(torch.int32)

    def vp(t):
        return ctypes.c_void_p(t.data_ptr())

    def run(fn, what=""):
        print("sweep:", what, file=sys.stderr, flush=True)
        fn()  # warm (tables, pool)
        torch.cuda.synchronize()
        ctx.profile(True)
        fn()
        rep = ctx.profile_report()
        ctx.profile(False)
        rep.pop("phases", None)
        rep.pop("kernels_by_phase", None)
        rep.pop("timeline", None)
        merge_lde(rep)
        return rep

    def emit(kind, kernel, rep, **kw):
        v = rep.get(kernel)
        if not v:
            return
        ms = v["ms"]
        line = {"sweep": kind, "kernel": kernel, "launches": v["launches"], "ms": round(ms, 4), **kw}
        if v["bytes"]:
            gbs = v["bytes"] / (ms * 1e-3) / 1e9
            line.update({"GB/s": round(gbs, 1), "hbm_frac": round(gbs / hbm, 4)})
        if v["perms"]:
            line["Gperm/s"] = round(v["perms"] / (ms * 1e-3) / 1e9, 3)
        print(json.dumps(line), flush=True)

    def check(rc):
        if rc != 0:
            raise RuntimeError(L.lg_last_error(ctx.h).decode())

    only = [w for w in a.sweep_only.split(",") if w]

    def want(kind, log):
        return not only or kind in only or f"{kind}:{log}" in only

    for log_out, cols in [(16, 1024), (18, 512), (20, 256), (22, 128), (24, 64)]:
        if not want("lde", log_out):
            continue
        n = 1 << (log_out - 2)
        x = field(n * cols)
        y = torch.empty(4 * n * cols, dtype=torch.int32, device=dev)
        rep = run(lambda: check(L.lg_rs_encode(ctx.h, vp(x), n, cols, vp(y), 1)), f"lde {log_out} {cols}")
        emit("lde", "lde", rep, rows_out=1 << log_out, cols=cols)
        del x, y
    for log_out, cols in [(16, 256), (20, 64), (22, 16)]:
        if not want("commit", log_out):
            continue
        n = 1 << (log_out - 2)
        x = field(n * cols)
        ptrs = (ctypes.c_void_p * cols)(*[x.data_ptr() + 4 * n * i for i in range(cols)])
        rows = (ctypes.c_uint64 * 1)(n)
        nb, ne = (ctypes.c_uint32 * 1)(cols), (ctypes.c_uint32 * 1)(0)
        root = (ctypes.c_uint32 * 8)()
        rep = run(lambda: check(L.lg_commit_root(ctx.h, 1, rows, nb, ne, ptrs, 1, root)), f"commit {log_out} {cols}")
        for k in ("lde", "hash_leaves", "merkle_level", "merkle_tail", "merkle_inject"):
            emit("merkle_commit", k, rep, rows_out=1 << log_out, cols=cols)
        del x
    alpha = (ctypes.c_uint32 * 6)(*[12345 + i for i in range(6)])
    for logn in (18, 20, 22, 24):
        if not want("fold", logn):
            continue
        n = 1 << logn
        x = field(6 * n)
        y = torch.empty(3 * n, dtype=torch.int32, device=dev)
        rep = run(lambda: check(L.lg_fri_fold(ctx.h, vp(x), n, alpha, vp(y), 1)), f"fold {logn}")
        emit("fri_fold", "fri_fold", rep, n_e6=n)
        del x, y
    for logr, cols in [(20, 256), (22, 64)]:
        if not want("deep", logr):
            continue
        rows = 1 << logr
        x = field(rows * cols)
        vals = field(6 * cols)
        out = torch.empty(6 * rows, dtype=torch.int32, device=dev)
        z = (ctypes.c_uint32 * 6)(*[777 + i for i in range(6)])
        rep = run(lambda: check(L.lg_deep_quotient(ctx.h, vp(x), cols, rows, alpha, z, vp(vals), vp(out), 1)),
                  f"deep {logr} {cols}")
        emit("deep", "deep", rep, rows=rows, cols=cols)
        del x, out
    ctx.close()


def max_over_ranks(values, dist, device):
    """Element-wise maximum of per-rank values: a job of N replicas takes as
    long as its slowest rank.  Identity with one process."""
    if dist is None:
        return [float(v) for v in values]
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t]


# ---------------------------------------------------------------------- GPU arm
def device_idle(timeline, phase_names):
    """Gaps between the recorded launches of one prove on its stream (device
    time with no recorded kernel running), total and per prove phase (a gap
    counts in the phase of the launch that ends it).  Small unrecorded
    kernels and copies fall inside gaps."""
    spans = sorted((t0, t0 + ms, ph) for (_, ph, t0, ms) in timeline)
    if not spans:
        return None
    by, end, total = {}, spans[0][1], 0.0
    for t0, t1, ph in spans[1:]:
        if t0 > end:
            gap = t0 - end
            total += gap
            name = phase_names[ph] if ph < len(phase_names) else "after last phase"
            by[name] = by.get(name, 0.0) + gap
        end = max(end, t1)
    return {"total": round(total, 3), "span": round(end - spans[0][0], 3),
            "by_phase": {k: round(v, 3) for k, v in by.items()}}


def main():
    a = parse()
    if a.sweep:
        return sweep(a)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if a.impl == "reference":
        return reference_arm(a, rank)

    import numpy as np
    import torch
    from loom_b200 import Context, field as F, plonk, proof

    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    device = local
    torch.cuda.set_device(device)

    comp, wit = plonk.build(a.instances, 1 << a.log_n, seed=0x10AD + rank)
    mont = [np.ascontiguousarray(F.to_mont(w)) for w in wit]
    dev_cols = [torch.from_numpy(m.view(np.int32)).to(f"cuda:{device}") for m in mont]
    dev_ptrs = [t.data_ptr() for t in dev_cols]
    # pinned host witness, columns back to back in descriptor order (one copy)
    pinned_all = torch.empty(sum(m.size for m in mont), dtype=torch.int32, pin_memory=True)
    host_all = pinned_all.numpy().view(np.uint32)
    host_cols, off = [], 0
    for m in mont:
        host_all[off:off + m.size] = m
        host_cols.append(host_all[off:off + m.size])
        off += m.size
    h2d_bytes = int(sum(m.nbytes for m in mont))
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{device}")  # > 126 MB L2
    torch.cuda.synchronize()

    ctx = Context(device)
    tune = None
    if not a.no_tune:
        from loom_b200 import autotune as AT
        tune = AT.autotune(ctx, force=a.retune)
    tparams = tune["params"] if tune else None

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(max(a.warmup, 3)):
        pb = ctx.prove(comp.words, dev_ptrs, a.queries, on_device=True)
    p = proof.decode(pb)
    assert all(v == p.final_poly[0] for v in p.final_poly), "final FRI polynomial is not constant"

    # ---- timed: witness resident in HBM
    # Python's cyclic garbage collector stays off through the timed loops: a
    # full collection of this process's heap, triggered by the few objects a
    # call allocates, stalled single steps by up to hundreds of milliseconds
    gc.collect()
    gc.disable()
    barrier()
    clocks = ClockSampler(device)
    clocks.start()
    launches0 = ctx.kernel_launches()
    times = []
    # the caller's proof buffer, written in place; page-locked, so the proof's
    # per-query sections arrive by DMA straight from the device
    out = torch.empty(2 * len(pb), dtype=torch.uint8, pin_memory=True).numpy()
    for _ in range(a.steps):
        flush.fill_(1)
        torch.cuda.synchronize()
        ctx.mark(0)
        n = ctx.prove_into(out, comp.words, dev_ptrs, a.queries, on_device=True)
        ctx.mark(1)
        times.append(ctx.elapsed_ms(0, 1))
    pb = bytes(out[:n])
    launches = ctx.kernel_launches() - launches0
    # ---- timed: host buffers in, proof bytes out (public API end to end)
    for _ in range(max(a.warmup, 3)):  # warm the host-buffer path as the device path was
        ctx.prove_into(out, comp.words, host_cols, a.queries, on_device=False)
    e2e_times = []
    for _ in range(a.steps):
        flush.fill_(1)
        torch.cuda.synchronize()
        ctx.mark(2)
        n = ctx.prove_into(out, comp.words, host_cols, a.queries, on_device=False)
        ctx.mark(3)
        e2e_times.append(ctx.elapsed_ms(2, 3))
    pbh = bytes(out[:n])
    # ---- timed: the plain per-kernel prover (one launch per group / module)
    ctx.set_batched(False)
    ctx.prove(comp.words, dev_ptrs, a.queries, on_device=True)
    plain_times = []
    for _ in range(a.steps):
        flush.fill_(1)
        torch.cuda.synchronize()
        ctx.mark(4)
        n = ctx.prove_into(out, comp.words, dev_ptrs, a.queries, on_device=True)
        ctx.mark(5)
        plain_times.append(ctx.elapsed_ms(4, 5))
    pbp = bytes(out[:n])
    ctx.set_batched(True)
    clk = clocks.stop()
    gc.enable()
    barrier()
    assert pbh == pb, "host-buffer and device-buffer proofs differ"
    assert pbp == pb, "plain and batched proofs differ"
    # max over ranks now, before the sections only rank 0 runs (every rank
    # takes the same collective steps in the same order)
    ms, e2e_ms, plain_ms = max_over_ranks(
        [statistics.mean(times), statistics.mean(e2e_times), statistics.mean(plain_times)], dist, f"cuda:{device}")

    # ---- throughput: several proofs in flight, one context + stream each
    from loom_b200.pool import ProverPool
    thr = []
    gc.collect()
    gc.disable()  # as in the timed loops above
    for S in [int(x) for x in a.streams.split(",") if x]:
        with ProverPool(S, device, tparams) as pool:
            for _ in range(2):  # warm every context (buffers, pools, tables), twice
                for f in [pool.submit(comp.words, dev_ptrs, a.queries, on_device=True) for _ in range(S)]:
                    f.result()
            jobs = S * max(4, a.steps)
            walls = []
            for _ in range(3):  # median of three batches: one host stall does not set the figure
                flush.fill_(1)
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                futs = [pool.submit(comp.words, dev_ptrs, a.queries, on_device=True) for _ in range(jobs)]
                outs = [f.result() for f in futs]
                e1.record()
                torch.cuda.synchronize()
                assert all(o == pb for o in outs), "concurrent proofs differ from the single-stream proof"
                del outs, futs
                walls.append(e0.elapsed_time(e1))
            wall = statistics.median(walls)
            thr.append({"streams": S, "proofs": jobs, "ms": round(wall, 3), "proofs_per_s": round(jobs * 1e3 / wall, 3),
                        "ms_each_batch": [round(w, 3) for w in walls]})
    gc.enable()

    # ---- batched form: 40 modules of uneven sizes (log2 rows 10-20, seeded)
    # with plonk gates, a copy constraint and a range lookup into a shared 2^8
    # table; batched against plain on the same inputs, byte-identical proofs
    c4 = None
    if not a.no_c4 and world == 1:
        sizes = plonk.mixed_sizes(40, 10, 20, 0xC4)
        c4comp, c4wit = plonk.build_mixed(sizes, seed=0xC4)
        c4dev = [torch.from_numpy(F.to_mont(w).astype(np.int64)).to(torch.int32).to(f"cuda:{device}") for w in c4wit]
        c4ptrs = [t.data_ptr() for t in c4dev]
        c4out = torch.empty(64 << 20, dtype=torch.uint8, pin_memory=True).numpy()
        res4 = {}
        for mode in ("batched", "plain"):
            ctx.set_batched(mode == "batched")
            for _ in range(2):
                n4 = ctx.prove_into(c4out, c4comp.words, c4ptrs, a.queries, on_device=True)
            ts = []
            for _ in range(max(2, min(a.steps, 3))):
                flush.fill_(1)
                torch.cuda.synchronize()
                ctx.mark(8)
                n4 = ctx.prove_into(c4out, c4comp.words, c4ptrs, a.queries, on_device=True)
                ctx.mark(9)
                ts.append(ctx.elapsed_ms(8, 9))
            res4[mode] = (statistics.mean(ts), bytes(c4out[:n4]))
        ctx.set_batched(True)
        p4 = proof.decode(res4["batched"][1])
        bus = [0] * 6
        for ents in p4.exposed.values():
            for (_, _, e) in ents:
                bus = [(x + y) % F.P for x, y in zip(bus, e)]
        c4 = {"workload": "40 modules, log2 rows 10-20 (seeded), plonk gates + copy constraint + range lookup "
                          "into a 2^8 table, Poseidon2, %d queries" % a.queries,
              "rows": int(sum(1 << x for x in sizes)), "log2_rows": sizes,
              "batched_ms": round(res4["batched"][0], 3), "plain_ms": round(res4["plain"][0], 3),
              "batched_speedup_vs_plain": round(res4["plain"][0] / res4["batched"][0], 3),
              "proofs_identical": res4["batched"][1] == res4["plain"][1],
              "final_poly_constant": all(v == p4.final_poly[0] for v in p4.final_poly),
              "logup_bus_balanced": bus == [0] * 6}
        del c4dev

    # ---- the same workload with the circuit constants (selectors, copy
    # permutation, identity columns) as setup columns precommitted once
    # (setup.Setup): each proof commits only the wires and the grand product
    # ---- verification of the headline proof (lg_verify: host transcript and
    # checks, Merkle openings and DEEP bridge on the GPU)
    ctx.verify(comp.words, pb, a.queries)
    vts = []
    for _ in range(3):
        t0 = time.perf_counter()
        ctx.verify(comp.words, pb, a.queries)
        vts.append((time.perf_counter() - t0) * 1e3)
    verify_res = {"ms": round(statistics.median(vts), 3), "accepted": True, "proof_bytes": len(pb)}

    setup_res = None
    if world == 1:
        scomp, swit, sset = plonk.build_with_setup(a.instances, 1 << a.log_n, seed=0x10AD)
        sdev = [torch.from_numpy(F.to_mont(w).astype(np.int64)).to(torch.int32).to(f"cuda:{device}") for w in swit]
        sptrs = [t.data_ptr() for t in sdev]
        sset_d = [torch.from_numpy(F.to_mont(w).astype(np.int64)).to(torch.int32).to(f"cuda:{device}") for w in sset]
        torch.cuda.synchronize()
        ctx.mark(8)
        ctx.setup(scomp.words, [t.data_ptr() for t in sset_d], on_device=True)
        ctx.mark(9)
        setup_ms = ctx.elapsed_ms(8, 9)
        sout = torch.empty(2 * len(pb), dtype=torch.uint8, pin_memory=True).numpy()
        for _ in range(2):
            ctx.prove_into(sout, scomp.words, sptrs, a.queries, on_device=True)
        ts = []
        for _ in range(max(3, a.steps)):
            flush.fill_(1)
            torch.cuda.synchronize()
            ctx.mark(8)
            ns = ctx.prove_into(sout, scomp.words, sptrs, a.queries, on_device=True)
            ctx.mark(9)
            ts.append(ctx.elapsed_ms(8, 9))
        ps = proof.decode(bytes(sout[:ns]))
        setup_res = {"workload": "the prove workload with QL..QK, sigma_k and ID_k as setup columns",
                     "setup_ms": round(setup_ms, 3), "prove_ms": round(statistics.mean(ts), 3),
                     "vs_all_witness_ms": round(ms, 3), "proof_bytes": ns,
                     "final_poly_constant": all(v == ps.final_poly[0] for v in ps.final_poly)}
        del sdev, sset_d

    # ---- serving: requests of mixed sizes (log2 rows 12-20, 1-8 instances) with
    # Poisson arrivals, admitted by HBM budget, overlapping on the GPU
    serve_res = None
    if a.serve_requests > 0 and world == 1:
        from loom_b200 import serve as SV
        rng = np.random.Generator(np.random.PCG64(0x5E4E))
        shapes = [(int(rng.integers(12, 21)), int(rng.integers(1, 9))) for _ in range(a.serve_shapes)]
        pool_reqs = [SV.make_request(i, lg, inst, a.queries, seed=0x77 + i) for i, (lg, inst) in enumerate(shapes)]
        # sequential plain-GPU proving of each shape once (the comparison baseline)
        pctx = Context(device, tparams)
        pctx.set_batched(False)
        plain_one = []
        ref_proof = {}
        for r in pool_reqs:
            pctx.prove(r.words, r.witness, r.num_queries)  # warm
            pctx.mark(6)
            ref_proof[r.rid] = pctx.prove(r.words, r.witness, r.num_queries)
            pctx.mark(7)
            plain_one.append(pctx.elapsed_ms(6, 7))
        pctx.close()
        sweeps = []
        for rate in [float(x) for x in a.serve_rate.split(",") if x]:
            reqs = []
            for i in range(a.serve_requests):
                t = pool_reqs[i % len(pool_reqs)]
                reqs.append(SV.Request(i, t.words, t.witness, t.num_queries, t.rows))
            shape_of = {i: i % len(pool_reqs) for i in range(a.serve_requests)}
            res = SV.serve(reqs, SV.poisson_arrivals(len(reqs), rate, 11), streams=a.serve_streams, device=device,
                           warm=pool_reqs, tuning=tparams)
            same = all(r.proof == ref_proof[shape_of[r.rid]] for r in res["finished"])
            seq_ms = sum(plain_one[shape_of[i]] for i in range(a.serve_requests))
            sweeps.append({"rate_per_s": rate, "requests": res["requests"], "p50_ms": round(res["p50_ms"], 2),
                           "p99_ms": round(res["p99_ms"], 2), "proofs_per_s": round(res["proofs_per_s"], 2),
                           "errors": res["errors"], "first_error": res["first_error"],
                           "proofs_identical_to_alone": same,
                           "measured_need_mb": [round(x / 2**20, 1) for x in res["measured_need_bytes"]],
                           "admissions_deferred_for_memory": res["admissions_deferred_for_memory"]})
        serve_res = {"shapes": [{"log_rows": lg, "instances": ins} for lg, ins in shapes],
                     "streams": a.serve_streams, "queries": a.queries,
                     "sequential_plain_proofs_per_s": round(len(plain_one) * 1e3 / sum(plain_one), 2),
                     "plain_ms_per_shape": [round(x, 2) for x in plain_one],
                     "sweep": sweeps}

    # ---- per-kernel events over a profiled step (roofline of the dominant kernel)
    flush.fill_(1)
    torch.cuda.synchronize()
    ctx.profile(True)
    ctx.prove(comp.words, dev_ptrs, a.queries, on_device=True)
    rep = ctx.profile_report()
    ctx.profile(False)
    phases = rep.pop("phases", {})
    by_phase = rep.pop("kernels_by_phase", {})
    idle = device_idle(rep.pop("timeline", []), list(phases))
    merge_lde(rep)

    if rank == 0:
        peaks = {}
        try:
            with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
                peaks = json.load(f)
        except OSError:
            pass
        hbm = peaks.get("hbm_gbs")
        hbm_src = "measured" if hbm else "fallback"
        hbm = hbm or 6650.0
        total_k = sum(v["ms"] for v in rep.values()) or 1.0
        hbm_kernels = ("lde", "coset_eval", "quotient_intt", "deep", "fri_fold", "quotient_eval")
        p2_kernels = ("hash_leaves", "merkle_inject", "merkle_level")
        shares = {k: round(v["ms"] / total_k, 4) for k, v in rep.items()}
        dom = max(rep, key=lambda k: rep[k]["ms"]) if rep else None
        traffic = {}
        try:
            with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
                traffic = json.load(f)
        except OSError:
            pass

        def traffic_of(k, per):
            # DRAM bytes per launch from an ncu capture, as a ratio to the
            # algorithmic bytes of the captured launch
            t = traffic.get(k)
            if isinstance(t, dict) and "dram_bytes_per_algorithmic_byte" in t:
                return round(t["dram_bytes_per_algorithmic_byte"] * per)
            return t

        def hbm_roof(k):
            v = rep[k]
            per = v["bytes"] / v["launches"]
            ach = per / (v["ms"] / v["launches"] * 1e-3) / 1e9
            return {"kernel": k, "bound": "hbm", "achieved": round(ach, 1), "peak": hbm, "unit": "GB/s",
                    "frac": round(ach / hbm, 4), "peak_source": hbm_src,
                    "traffic": traffic_of(k, per), "algorithmic_bytes_per_launch": round(per),
                    "avg_launch_ms": round(v["ms"] / v["launches"], 5), "share": shares[k]}

        # Poseidon2 kernels: integer-multiply bound; 834 field products per
        # width-24 permutation, 4 IMAD each = 3336 IMAD per permutation.
        sm_count = torch.cuda.get_device_properties(device).multi_processor_count
        clk_mhz = clk.get("sm_mhz") or peaks.get("sm_max_mhz") or 1965.0
        imad_peak = sm_count * 64 * clk_mhz * 1e6
        p2 = {k: rep[k] for k in p2_kernels if k in rep}
        p2_ms = sum(v["ms"] for v in p2.values())
        p2_perms = sum(v["perms"] for v in p2.values())
        p2_roof = None
        if p2_ms:
            ach = p2_perms / (p2_ms * 1e-3)
            p2_roof = {"kernels": list(p2), "bound": "int32", "achieved": round(ach / 1e9, 3),
                       "peak": round(imad_peak / 3336 / 1e9, 3), "unit": "Gperm/s",
                       "frac": round(ach / (imad_peak / 3336), 4),
                       "peak_source": f"nominal {sm_count} SMs x 64 IMAD/clk at the sampled {clk_mhz:.0f} MHz",
                       "share": round(p2_ms / total_k, 4)}
        hbm_dom = max((k for k in rep if k in hbm_kernels), key=lambda k: rep[k]["ms"], default=None)
        roof = hbm_roof(hbm_dom) if hbm_dom else None
        # every HBM-bound kernel of the prove, not only the dominant one
        rooflines = {k: {kk: hbm_roof(k)[kk] for kk in ("achieved", "frac", "avg_launch_ms", "share")}
                     for k in hbm_kernels if k in rep and rep[k]["bytes"] > 0}
        base = None
        if world == 1 and not a.no_cpu_baseline:
            base = cpu_baseline(a, steps=max(1, a.cpu_steps), warmup=1)
        line = {
            "metric": METRIC, "value": round(ms, 3), "unit": "ms", "n_gpus": world, "steps": a.steps,
            "warmup": max(a.warmup, 3), "ms_per_step": round(ms, 3), "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded plonk-like witnesses)",
            "config": {"workload": workload_name(a), "instances": a.instances, "log_rows": a.log_n,
                       "queries": a.queries, "mode": "batched", "parallelism": f"replicas x{world}",
                       "l2": "flushed between steps (256 MB write)"},
            "proofs_per_s": round(world * 1e3 / ms, 3),
            "plain": {"value": round(plain_ms, 3), "unit": "ms",
                      "note": "same kernels, one launch per group / module (the plain per-kernel prover)"},
            "batched_speedup_vs_plain": round(plain_ms / ms, 3),
            "throughput": thr,
            "serve": serve_res,
            "best_throughput_vs_plain": round(max([t["proofs_per_s"] for t in thr] + [1e3 / ms]) * plain_ms / 1e3, 3),
            "e2e": {"value": round(e2e_ms, 3), "unit": "ms",
                    "median_ms": round(statistics.median(e2e_times), 3), "min_ms": round(min(e2e_times), 3),
                    "note": "value: mean over the timed steps (rank 0's steps for median and min)",
                    "h2d_bytes_per_step": h2d_bytes,
                    "d2h_bytes_per_step": len(pbh)},
            "gpu_launches": int(launches),
            "roofline": roof,
            "rooflines_hbm": rooflines,
            "roofline_poseidon2": p2_roof,
            "kernel_shares": shares,
            "kernel_ms_profiled_step": round(total_k, 3),
            "host_phases_ms": {k: round(v, 3) for k, v in phases.items()},
            "step_ms": {"prove": [round(x, 3) for x in times], "e2e": [round(x, 3) for x in e2e_times],
                        "plain": [round(x, 3) for x in plain_times]},
            "c4_mixed_lookup": c4,
            "setup_precommit": setup_res,
            "verify": verify_res,
            "tuning": tune,
            "kernel_ms_by_phase": {ph: {k: round(v["ms"], 3) for k, v in ks.items()} for ph, ks in by_phase.items()},
            "device_idle_ms": idle,
            "dominant_kernel": dom,
            "cpu_baseline": base,
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
