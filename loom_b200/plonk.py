"""Seeded synthetic plonk-like workloads (the prove benchmark's inputs).

Each instance i is one module "plonk_i" of N rows with base columns
L_i, R_i, O_i (wires a, b, c) and QL_i, QR_i, QM_i, QO_i, QK_i (selectors),
named as the reference benchmark names them (bench/main.go:86-106,
integration_test/gnark_plonk/plonk_gnark_utils.go:221-233).  The gate is
QL.L + QR.R + QM.L.R + QO.O + QK = 0 and a copy constraint covers the three
wires (arguments.CopyConstraint).

Witness: a and b uniform in [0, p); selectors are seeded 0/1 patterns; c is
solved so every gate holds (QO = 1 wherever another selector is set).  The
copy permutation links positions that hold equal values: random cycles of
length 2..4 over the a/b positions (their values made equal), c positions
fixed points.  Everything is deterministic in (seed, instance).
"""
from __future__ import annotations

from typing import Dict, List, Tuple

import numpy as np

from . import field as F
from .program import Builder, Compiled, Module, col, copy_constraint, range_check


def _ith(s: str, i: int) -> str:
    return f"{s}_{i}"


def instance_witness(n: int, seed: int, instance: int) -> Tuple[Dict[str, np.ndarray], np.ndarray]:
    rng = np.random.Generator(np.random.PCG64([seed, instance]))
    a = rng.integers(0, F.P, n, dtype=np.uint64)
    b = rng.integers(0, F.P, n, dtype=np.uint64)
    ql, qr, qm, qc = (rng.integers(0, 2, n, dtype=np.uint64) for _ in range(4))
    any_sel = (ql | qr | qm | qc) > 0
    qo = np.where(any_sel, 1, rng.integers(0, 2, n, dtype=np.uint64)).astype(np.uint64)
    # copy cycles over a/b positions (0..2n-1), values equalised along each cycle
    S = np.arange(3 * n, dtype=np.int64)
    vals = np.concatenate([a, b])
    perm = rng.permutation(2 * n)
    pos, covered = 0, int(n)  # link about half of the a/b positions
    while pos < covered:
        k = int(rng.integers(2, 5))
        cyc = perm[pos:pos + k]
        pos += k
        if len(cyc) < 2:
            break
        vals[cyc] = vals[cyc[0]]
        for j in range(len(cyc)):
            S[cyc[j]] = cyc[(j + 1) % len(cyc)]
    a, b = vals[:n], vals[n:]
    p = np.uint64(F.P)
    lin = (ql * a % p + qr * b % p + (qm * (a * b % p)) % p + qc) % p
    c = np.where(qo == 1, (p - lin) % p, rng.integers(0, F.P, n, dtype=np.uint64))
    # rows with qo == 0 have no other selector set, so the gate is 0 there
    cols = {
        _ith("L", instance): a, _ith("R", instance): b, _ith("O", instance): c,
        _ith("QL", instance): ql, _ith("QR", instance): qr, _ith("QM", instance): qm,
        _ith("QO", instance): qo, _ith("QK", instance): qc,
    }
    return {k: v.astype(np.uint32) for k, v in cols.items()}, S


def build(n_instances: int, n: int, seed: int = 0x10AD) -> Tuple[Compiled, List[np.ndarray]]:
    """Program and witness (canonical values, descriptor order) of
    `n_instances` plonk-like modules of `n` rows."""
    b = Builder()
    trace: Dict[str, np.ndarray] = {}
    for i in range(n_instances):
        m = Module(_ith("plonk", i), n)
        L, R, O = col(_ith("L", i)), col(_ith("R", i)), col(_ith("O", i))
        QL, QR, QM, QO, QK = (col(_ith(s, i)) for s in ("QL", "QR", "QM", "QO", "QK"))
        m.assert_zero(QL * L + QR * R + QM * L * R + QO * O + QK)
        b.add_module(m)
        w, S = instance_witness(n, seed, i)
        trace.update(w)
        copy_constraint(b, m.name, [L, R, O], S, _ith("plonk.S", i))
    trace.update(b.generated)
    compiled = b.compile()
    witness = [np.ascontiguousarray(trace[name], dtype=np.uint32) for (name, fld, rows) in compiled.witness_columns]
    return compiled, witness


def build_with_setup(n_instances: int, n: int, seed: int = 0x10AD):
    """The plonk program of build() with its circuit constants as setup columns
    (expr.Setup): the selectors QL..QK, the copy permutation sigma_k and the
    identity columns ID_k, precommitted once (setup/setup.go:68-124) instead of
    committed in every proof.  Returns (program, witness, setup values), each
    list in descriptor order."""
    b = Builder()
    trace: Dict[str, np.ndarray] = {}
    for i in range(n_instances):
        m = Module(_ith("plonk", i), n)
        L, R, O = col(_ith("L", i)), col(_ith("R", i)), col(_ith("O", i))
        QL, QR, QM, QO, QK = (col(_ith(s, i)) for s in ("QL", "QR", "QM", "QO", "QK"))
        m.assert_zero(QL * L + QR * R + QM * L * R + QO * O + QK)
        b.add_module(m)
        w, S = instance_witness(n, seed, i)
        trace.update(w)
        copy_constraint(b, m.name, [L, R, O], S, _ith("plonk.S", i))
        b.mark_setup(*(_ith(s, i) for s in ("QL", "QR", "QM", "QO", "QK")))
        b.mark_setup(*(m.id_support_name(k) for k in range(3)), *(f"{_ith('plonk.S', i)}_{k}" for k in range(3)))
    trace.update(b.generated)
    compiled = b.compile()
    witness = [np.ascontiguousarray(trace[name], dtype=np.uint32) for (name, fld, rows) in compiled.witness_columns]
    setup = [np.ascontiguousarray(trace[name], dtype=np.uint32) for (name, fld, rows) in compiled.setup_columns]
    return compiled, witness, setup


def build_mixed(log_sizes: List[int], seed: int = 0x10AD, range_bound: int = 256) -> Tuple[Compiled, List[np.ndarray]]:
    """Modules of uneven sizes 2^log_sizes[i], each a plonk-like module as in
    build() plus a column RC_i of values in [0, range_bound) range-checked by a
    logup lookup into the shared range table (arguments.Range): the batched
    form of the prove benchmark (gates, a permutation argument and a lookup)."""
    b = Builder()
    trace: Dict[str, np.ndarray] = {}
    for i, lg in enumerate(log_sizes):
        n = 1 << lg
        m = Module(_ith("plonk", i), n)
        L, R, O = col(_ith("L", i)), col(_ith("R", i)), col(_ith("O", i))
        QL, QR, QM, QO, QK = (col(_ith(s, i)) for s in ("QL", "QR", "QM", "QO", "QK"))
        m.assert_zero(QL * L + QR * R + QM * L * R + QO * O + QK)
        b.add_module(m)
        w, S = instance_witness(n, seed, i)
        trace.update(w)
        copy_constraint(b, m.name, [L, R, O], S, _ith("plonk.S", i))
        rng = np.random.Generator(np.random.PCG64([seed, i, 0x5243]))
        trace[_ith("RC", i)] = rng.integers(0, range_bound, n, dtype=np.uint32)
        range_check(b, col(_ith("RC", i)), m.name, range_bound)
    trace.update(b.generated)
    compiled = b.compile()
    witness = [np.ascontiguousarray(trace[name], dtype=np.uint32) for (name, fld, rows) in compiled.witness_columns]
    return compiled, witness


def build_with_ratio(n: int, seed: int = 5, permuted: bool = True):
    """A plonk module next to a module with columns A and B (staged at
    RoundFold) and the running ratio of (A - gamma) / (B - gamma) at
    RoundRunningSums (board/product.go:72-198).  With B a permutation of A the
    exposed end is 1.  Returns (program, witness, name of the exposed end)."""
    from .program import ROUND_FOLD, ROUND_LOG_DERIVATIVE, ROUND_RUNNING_SUMS, coin
    rng = np.random.Generator(np.random.PCG64([seed, 0x5252]))
    b = Builder()
    trace: Dict[str, np.ndarray] = {}
    m0 = Module("plonk_0", n)
    L, R, O = col("L_0"), col("R_0"), col("O_0")
    QL, QR, QM, QO, QK = (col(f"{s}_0") for s in ("QL", "QR", "QM", "QO", "QK"))
    m0.assert_zero(QL * L + QR * R + QM * L * R + QO * O + QK)
    b.add_module(m0)
    w, S = instance_witness(n, seed, 0)
    trace.update(w)
    copy_constraint(b, "plonk_0", [L, R, O], S, "plonk.S_0")
    b.add_module(Module("ratio_0", n))
    a = rng.integers(0, F.P, n, dtype=np.uint64).astype(np.uint32)
    trace["A_0"] = a
    trace["B_0"] = rng.permutation(a) if permuted else rng.integers(0, F.P, n, dtype=np.uint64).astype(np.uint32)
    b.stage_leaves(ROUND_FOLD, col("A_0"), col("B_0"))
    gamma = coin(ROUND_LOG_DERIVATIVE)
    end = b.add_running_ratio_step(ROUND_RUNNING_SUMS, "ratio_0", [col("A_0") - gamma], [col("B_0") - gamma],
                                   b.fresh_name("rr_"))
    b.product_buses.append([end])  # B is claimed to be a permutation of A: the end is one
    trace.update(b.generated)
    comp = b.compile()
    wit = [np.ascontiguousarray(trace[nm], dtype=np.uint32) for (nm, f, r) in comp.witness_columns]
    return comp, wit, end


def build_with_bus(n: int, seed: int = 9, balanced: bool = True):
    """A plonk module next to two modules joined by a width-2 bus
    (arguments.Bus, arguments/bus.go:42-67): "bussend_0" (n rows) sends the
    tuples (A0, A1) on the rows where SA = 1, "busrecv_0" (n/2 rows) receives
    (X0, X1) where SX = 1.  The received tuples are the sent ones in another
    order (one of them altered unless `balanced`); the unselected rows hold
    unrelated values.  Returns (program, witness, bus ends)."""
    from .program import bus
    rng = np.random.Generator(np.random.PCG64([seed, 0xB005]))
    b = Builder()
    trace: Dict[str, np.ndarray] = {}
    m0 = Module("plonk_0", n)
    L, R, O = col("L_0"), col("R_0"), col("O_0")
    QL, QR, QM, QO, QK = (col(f"{s}_0") for s in ("QL", "QR", "QM", "QO", "QK"))
    m0.assert_zero(QL * L + QR * R + QM * L * R + QO * O + QK)
    b.add_module(m0)
    w, S = instance_witness(n, seed, 0)
    trace.update(w)
    copy_constraint(b, "plonk_0", [L, R, O], S, "plonk.S_0")
    h = n // 2
    b.add_module(Module("bussend_0", n))
    b.add_module(Module("busrecv_0", h))
    rnd = lambda k: rng.integers(0, F.P, k, dtype=np.uint64).astype(np.uint32)
    a0, a1, x0, x1 = rnd(n), rnd(n), rnd(h), rnd(h)
    k = n // 4
    sa = np.zeros(n, dtype=np.uint32)
    sent = rng.choice(n, k, replace=False)
    sa[sent] = 1
    sx = np.zeros(h, dtype=np.uint32)
    recv = rng.choice(h, k, replace=False)
    sx[recv] = 1
    order = rng.permutation(k)
    x0[recv], x1[recv] = a0[sent][order], a1[sent][order]
    if not balanced:
        x1[recv[0]] = (int(x1[recv[0]]) + 1) % F.P
    trace.update({"A0_0": a0, "A1_0": a1, "SA_0": sa, "X0_0": x0, "X1_0": x1, "SX_0": sx})
    ends = bus(b, [col("SA_0")], [col("SX_0")], [([col("A0_0"), col("A1_0")], "bussend_0")],
               [([col("X0_0"), col("X1_0")], "busrecv_0")])
    trace.update(b.generated)
    comp = b.compile()
    wit = [np.ascontiguousarray(trace[nm], dtype=np.uint32) for (nm, f, r) in comp.witness_columns]
    return comp, wit, ends


def build_with_tuple_lookup(n: int, seed: int = 13, present: bool = True):
    """A plonk module next to a conditional tuple lookup
    (arguments.CLookupUnionTuple, arguments/lookup.go:86-110): the rows of
    (SA, SB) in "lookA_0" (n rows, selector SS) and of (XA, XB) in "lookB_0"
    (n/4 rows, selector SX) whose selector is non-zero lie among the rows of
    (TA, TB) in "table_0" (n/2 rows) whose selector ST is non-zero.  Selector
    values other than 1 weight the rows (a source row with SS = 2 counts twice;
    a target row with ST = 3 carries a third of its tuple's weight in its
    multiplicity); some target tuples repeat, one of them first on an
    unselected row.  Unless `present`, one selected source tuple is missing
    from the table.  Returns (program, witness)."""
    from .program import lookup_tuple
    rng = np.random.Generator(np.random.PCG64([seed, 0x7AB1]))
    b = Builder()
    trace: Dict[str, np.ndarray] = {}
    m0 = Module("plonk_0", n)
    L, R, O = col("L_0"), col("R_0"), col("O_0")
    QL, QR, QM, QO, QK = (col(f"{s}_0") for s in ("QL", "QR", "QM", "QO", "QK"))
    m0.assert_zero(QL * L + QR * R + QM * L * R + QO * O + QK)
    b.add_module(m0)
    w, S = instance_witness(n, seed, 0)
    trace.update(w)
    copy_constraint(b, "plonk_0", [L, R, O], S, "plonk.S_0")
    h, q = n // 2, n // 4
    for name, rows in (("table_0", h), ("lookA_0", n), ("lookB_0", q)):
        b.add_module(Module(name, rows))
    rnd = lambda k: rng.integers(0, F.P, k, dtype=np.uint64).astype(np.uint32)
    ta, tb = rnd(h), rnd(h)
    ta[5], tb[5] = ta[9], tb[9]        # a repeated tuple, both rows selected
    ta[2], tb[2] = ta[11], tb[11]      # repeated, first occurrence unselected
    st = (rng.integers(0, 4, h) > 0).astype(np.uint32)
    st[[5, 9, 11]] = 1
    st[2] = 0
    st[7] = 3
    live = np.flatnonzero(st)
    pick = lambda k: rng.choice(live, k)
    sa_idx, sx_idx = pick(n), pick(q)
    sa, sb, xa, xb = ta[sa_idx], tb[sa_idx], ta[sx_idx], tb[sx_idx]
    ss = (rng.integers(0, 3, n) > 0).astype(np.uint32)
    ss[[3, 4]] = 2
    sx = (rng.integers(0, 3, q) > 0).astype(np.uint32)
    junk = ss == 0
    sa[junk], sb[junk] = rnd(int(junk.sum())), rnd(int(junk.sum()))
    sa[0], sb[0], ss[0] = ta[7], tb[7], 1  # weight on the row whose selector is 3
    if not present:
        sb[1], ss[1] = (int(sb[1]) + 1) % F.P, 1
    trace.update({"TA_0": ta, "TB_0": tb, "ST_0": st, "SA_0": sa, "SB_0": sb, "SS_0": ss,
                  "XA_0": xa, "XB_0": xb, "SX_0": sx})
    lookup_tuple(b, [([col("SA_0"), col("SB_0")], "lookA_0"), ([col("XA_0"), col("XB_0")], "lookB_0")],
                 [([col("TA_0"), col("TB_0")], "table_0")], sel_s=[col("SS_0"), col("SX_0")], sel_t=[col("ST_0")])
    trace.update(b.generated)
    comp = b.compile()
    wit = [np.ascontiguousarray(trace[nm], dtype=np.uint32) for (nm, f, r) in comp.witness_columns]
    return comp, wit


def mixed_sizes(n_modules: int, lo: int, hi: int, seed: int) -> List[int]:
    """log2 module sizes drawn uniformly from [lo, hi] (seeded)."""
    rng = np.random.Generator(np.random.PCG64([seed, 0x5A5E]))
    return [int(x) for x in rng.integers(lo, hi + 1, n_modules)]


def check_gates(witness_by_name: Dict[str, np.ndarray], i: int) -> bool:
    g = lambda s: witness_by_name[_ith(s, i)].astype(np.uint64)
    p = np.uint64(F.P)
    v = (g("QL") * g("L") % p + g("QR") * g("R") % p + (g("QM") * (g("L") * g("R") % p)) % p
         + g("QO") * g("O") % p + g("QK")) % p
    return bool(np.all(v == 0))
