"""Host-side program builder: the part of loom's board/expr front end that the
Poseidon2 prove path consumes, compiled to this repository's flat program
descriptor (documented in include/loom_gpu.h).

It mirrors the reference's construction API so that a program built here is
the program the Go prover would build:
  * ``Expr`` / ``col`` / ``coin`` / ``const`` / ``fold``  — expr/ast.go,
    expr/utils.go:21-33 (Horner fold C0 + v(C1 + v(C2 + ...))).
  * ``Module.assert_zero`` / ``assert_zero_at`` / ``assert_equal_at`` —
    board/module.go:183-251 (Lagrange verifier columns "<module>.Lagrange_i").
  * ``Builder.stage_leaves`` / ``add_grand_product_step`` / ``fresh_name`` —
    board/rounds.go:108-135, board/board.go:66-69,251-267.
  * ``copy_constraint`` — arguments/permutation.go:37-127 (ID support and
    permutation columns generated as in board/module.go:229-293).
  * ``range_check`` / ``lookup`` — arguments/lookup.go:31-230: the range module
    and its column (board/module.go:56-71), lookup multiplicities
    (board/board.go:235-249) and cyclic logup columns with their exposed
    totals (board/logup.go:70-149).
  * ``Builder.compile`` — board/program.go:45-89 and the last-round sweep of
    board/rounds.go:219-292.
"""
from __future__ import annotations

from dataclasses import dataclass, field as dfield
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import field as F

ROUND_FOLD, ROUND_LOG_DERIVATIVE, ROUND_RUNNING_SUMS = 0, 1, 2
BASE, EXT = 0, 1
KIND_WITNESS, KIND_STEP, KIND_LAGRANGE, KIND_SETUP = 0, 1, 2, 3
OP_COL, OP_COIN, OP_CONST, OP_ADD, OP_SUB, OP_MUL, OP_EXPAVG, OP_EXPVAL = range(8)
STEP_GP, STEP_MULT, STEP_LOGUP, STEP_RATIO, STEP_MULTW = 0, 1, 2, 3, 4
MAGIC = 0x3150474C
RANGE_MODULE, LOGUP = "range", "logup"  # internal/constants/const.go:34,41
MAX_LOGUP_DEGREE, MAX_LOGUP_BATCH = 5, 4  # board/logup.go:37, arguments/lookup.go:156


class Expr:
    """Immutable expression tree over columns, round coins and constants."""

    __slots__ = ("op", "a", "b")

    def __init__(self, op, a=None, b=None):
        self.op, self.a, self.b = op, a, b

    def __add__(self, o): return Expr(OP_ADD, self, _lift(o))
    def __sub__(self, o): return Expr(OP_SUB, self, _lift(o))
    def __mul__(self, o): return Expr(OP_MUL, self, _lift(o))
    add = __add__
    sub = __sub__
    mul = __mul__

    def leaves(self) -> List["Expr"]:
        """Leaves in left-to-right order (expr/ast.go:602-639)."""
        if self.op in (OP_ADD, OP_SUB, OP_MUL):
            return self.a.leaves() + self.b.leaves()
        return [self]

    def key(self):
        if self.op == OP_COL:
            return ("c", self.a, self.b)
        if self.op == OP_COIN:
            return ("k", self.a)
        if self.op == OP_CONST:
            return ("v", self.a)
        if self.op == OP_EXPAVG:
            return ("x", self.a)
        if self.op == OP_EXPVAL:
            return ("e", self.a)
        return (self.op, self.a.key(), self.b.key())

    def degree(self) -> int:
        """expr Degree: columns (committed or verifier, exposed averages
        included) count 1, coins and constants 0."""
        if self.op in (OP_COL, OP_EXPAVG):
            return 1
        if self.op in (OP_COIN, OP_CONST, OP_EXPVAL):
            return 0
        if self.op == OP_MUL:
            return self.a.degree() + self.b.degree()
        return max(self.a.degree(), self.b.degree())


def _lift(o):
    return o if isinstance(o, Expr) else const(int(o))


def col(name: str, shift: int = 0) -> Expr:
    return Expr(OP_COL, name, int(shift))


def coin(r: int) -> Expr:
    """Round challenge "challenge@loom_r" (board/rounds.go:70-72)."""
    return Expr(OP_COIN, int(r))


def const(v: int) -> Expr:
    return Expr(OP_CONST, int(v) % F.P)


def exposed_average(total: str) -> Expr:
    """The constant extension column T/N of an exposed total T, N the size of
    the module using it (expr/ast.go:223-227)."""
    return Expr(OP_EXPAVG, total)


def exposed_value(name: str) -> Expr:
    """An exposed value as a constant; times L_0 it is the sparse verifier
    column expr.Exposed (board/product.go:109, the end P at row 0)."""
    return Expr(OP_EXPVAL, name)


def fold(v: Expr, cs: Sequence[Expr]) -> Expr:
    if not cs:
        return const(0)
    res = cs[-1]
    for c in reversed(cs[:-1]):
        res = c + (v * res)
    return res


def lagrange_name(module: str, i: int) -> str:
    return f"{module}.Lagrange_{i}"


@dataclass
class Module:
    name: str
    n: int
    relations: List[Expr] = dfield(default_factory=list)
    lagrange: Dict[str, int] = dfield(default_factory=dict)  # verifier column -> row

    def lagrange_col(self, i: int) -> Expr:
        nm = lagrange_name(self.name, i)
        self.lagrange[nm] = i
        return col(nm)

    def assert_zero(self, rel: Expr):
        self.relations.append(rel)

    def assert_zero_at(self, rel: Expr, *rows: int):
        disj = self.lagrange_col(rows[0])
        for r in rows[1:]:
            disj = disj + self.lagrange_col(r)
        self.assert_zero(rel * disj)

    def assert_zero_except_at(self, rel: Expr, *rows: int):
        """board/module.go:167-176 AssertZeroExceptAt: rel times the product
        of (1 - L_i) over the excepted rows."""
        conj = const(1) - self.lagrange_col(rows[0])
        for r in rows[1:]:
            conj = conj * (const(1) - self.lagrange_col(r))
        self.assert_zero(rel * conj)

    def assert_equal_at(self, a: Expr, b: Expr, i: int):
        self.assert_zero((a - b) * self.lagrange_col(i))

    def id_support_name(self, i: int) -> str:
        return f"{self.name}.ID_{i}_{self.n}"


@dataclass
class GrandProductStep:
    round: int
    module: str
    num: Expr
    den: Expr
    out: str


@dataclass
class MultiplicityStep:
    """board/board.go:235-249: one multiplicity column per target table."""
    round: int
    sources: List[Expr]
    targets: List[Expr]
    outs: List[str]


@dataclass
class TupleMultiplicityStep:
    """board/board.go:235-249 in general: tables of `width` expressions, with
    optional selectors (None: every row counts); one multiplicity column per
    target table."""
    round: int
    width: int
    sources: List[List[Expr]]
    targets: List[List[Expr]]
    sel_s: Optional[List[Expr]]
    sel_t: Optional[List[Expr]]
    outs: List[str]


@dataclass
class LogupStep:
    """board/logup.go:80-127: a cyclic logup column and its exposed total."""
    round: int
    module: str
    terms: List[Tuple[Expr, Expr]]  # (E, M): fraction M / E
    out: str
    total: str


@dataclass
class RunningRatioStep:
    """board/product.go:72-198: Z_i = prod_{k<=i} num_k / den_k, end P = Z_{N-1} exposed."""
    round: int
    module: str
    num: Expr
    den: Expr
    out: str
    end: str


@dataclass
class Compiled:
    words: np.ndarray              # descriptor, uint32
    witness_columns: List[Tuple[str, int, int]]  # (name, field, rows), in descriptor order
    modules: Dict[str, int]        # name -> N
    n_rounds: int
    logup_buses: List[List[str]] = dfield(default_factory=list)    # totals that sum to zero
    product_buses: List[List[str]] = dfield(default_factory=list)  # running-ratio ends whose product is one
    setup_columns: List[Tuple[str, int, int]] = dfield(default_factory=list)  # (name, field, rows), descriptor order


class Builder:
    def __init__(self):
        self.modules: Dict[str, Module] = {}
        self.rounds: List[dict] = []
        self.names = 0
        self.generated: Dict[str, np.ndarray] = {}  # generated base columns (ID support, permutation)
        self.logup_buses: List[List[str]] = []    # board.LogupBus (board/board.go:35-38)
        self.setup_names: set = set()             # expr.Setup columns (expr/ast.go:211-217)
        self.product_buses: List[List[str]] = []  # board.ProductBus (board/board.go:28-29)

    def add_module(self, m: Module):
        self.modules[m.name] = m

    def mark_setup(self, *names: str):
        """Declares columns as setup columns (expr.Setup, expr/ast.go:211-217):
        program constants precommitted once in the setup tree (setup/setup.go:68-124),
        never staged in a round."""
        self.setup_names.update(names)

    def fresh_name(self, prefix: str) -> str:
        self.names += 1
        return f"{prefix}{self.names}"

    def _grow(self, r: int):
        while len(self.rounds) <= r:
            self.rounds.append({"steps": [], "staged": []})

    def stage_columns(self, r: int, *names: str):
        self._grow(r)
        for n in names:
            if n not in self.rounds[r]["staged"]:
                self.rounds[r]["staged"].append(n)

    def stage_leaves(self, r: int, *exprs: Expr):
        for e in exprs:
            for lf in e.leaves():
                if lf.op == OP_COL and not self._is_verifier(lf.a):
                    self.stage_columns(r, lf.a)

    def _is_verifier(self, name: str) -> bool:
        return any(name in m.lagrange for m in self.modules.values())

    def add_lookup_multiplicity_step(self, r: int, S: Sequence[Expr], T: Sequence[Expr], output: str) -> List[str]:
        """Width-1 tables (board/board.go:235-249); outs "<output>_<i>"."""
        self._grow(r)
        outs = [f"{output}_{i}" for i in range(len(T))]
        self.rounds[r]["steps"].append(MultiplicityStep(r, list(S), list(T), outs))
        return outs

    def add_tuple_multiplicity_step(self, r: int, sel_s, sel_t, S: Sequence[Sequence[Expr]],
                                    T: Sequence[Sequence[Expr]], output: str) -> List[str]:
        """Tables of any width, with optional selectors (board/board.go:235-249,
        internal/poly/lookup_multiplicity.go:37-100); outs "<output>_<i>"."""
        widths = {len(t) for t in list(S) + list(T)}
        if len(widths) != 1:
            raise ValueError("lookup: inconsistent width")
        self._grow(r)
        outs = [f"{output}_{i}" for i in range(len(T))]
        self.rounds[r]["steps"].append(TupleMultiplicityStep(
            r, widths.pop(), [list(x) for x in S], [list(x) for x in T], None if sel_s is None else list(sel_s),
            None if sel_t is None else list(sel_t), outs))
        return outs

    def add_cyclic_logup_step(self, r: int, module: str, terms: Sequence[Tuple[Expr, Expr]], output: str) -> str:
        """board/logup.go:80-127: L - L_{-1} + T/N = sum_j M_j / E_j on every
        row (row 0 reads L_{N-1}); returns the exposed total's name."""
        if not terms:
            raise ValueError(f"logup {output}: no terms")
        if logup_constraint_degree(terms) > MAX_LOGUP_DEGREE:
            raise ValueError(f"logup {output}: constraint degree above {MAX_LOGUP_DEGREE}")
        total = output + "_total"
        self._grow(r)
        self.rounds[r]["steps"].append(LogupStep(r, module, list(terms), output, total))

        def prod_e(skip: int) -> Optional[Expr]:
            res = None
            for i, (e, _) in enumerate(terms):
                if i != skip:
                    res = e if res is None else res * e
            return res

        increment = col(output) - col(output, -1) + exposed_average(total)
        relation = increment * prod_e(-1)
        for j, (_, m) in enumerate(terms):
            num = m * prod_e(j) if len(terms) > 1 else m
            relation = relation - num
        self.modules[module].assert_zero(relation)
        return total

    def add_running_ratio_step(self, r: int, module: str, num: Sequence[Expr], den: Sequence[Expr], output: str) -> str:
        """board/product.go:72-121: Z·d·(1 - L_0 + E) - Z_{-1}·n = 0 and
        L_0·Z_{-1} - E = 0 with E = P·L_0, P the exposed end; returns P's name."""
        if not num and not den:
            raise ValueError(f"running ratio {output}: no factors")
        deg = running_ratio_constraint_degree(num, den)
        if deg > MAX_LOGUP_DEGREE:
            raise ValueError(f"running ratio {output}: constraint degree {deg} above {MAX_LOGUP_DEGREE}")

        def product(fs):
            res = None
            for f in fs:
                res = f if res is None else res * f
            return res

        end = output + "_end"
        pn, pd = product(num), product(den)
        self._grow(r)
        self.rounds[r]["steps"].append(RunningRatioStep(r, module, pn if pn is not None else const(1),
                                                        pd if pd is not None else const(1), output, end))
        m = self.modules[module]
        z, zprev = col(output), col(output, -1)
        l0 = m.lagrange_col(0)
        e = exposed_value(end) * l0
        lhs = z * (const(1) - l0 + e)
        if pd is not None:
            lhs = lhs * pd
        rhs = zprev if pn is None else zprev * pn
        m.assert_zero(lhs - rhs)
        m.assert_zero(l0 * zprev - e)
        return end

    def add_grand_product_step(self, r: int, module: str, num: Expr, den: Expr, out: str):
        self._grow(r)
        self.rounds[r]["steps"].append(GrandProductStep(r, module, num, den, out))
        m = self.modules[module]
        gp, gps = col(out), col(out, 1)
        m.assert_zero(gps * den - gp * num)
        m.assert_zero_at(gp - const(1), 0)

    # ------------------------------------------------------------------ compile
    def compile(self) -> Compiled:
        if not self.rounds:
            self.rounds = [{"steps": [], "staged": []}]
        n_rounds = len(self.rounds)
        verifier = {nm: (mname, row) for mname, m in self.modules.items() for nm, row in m.lagrange.items()}
        owner: Dict[str, str] = {}
        for mname, m in self.modules.items():
            for rel in m.relations:
                for lf in rel.leaves():
                    if lf.op == OP_COL and lf.a not in verifier:
                        owner[lf.a] = mname
        step_out = {}
        for rd in self.rounds:
            for s_ in rd["steps"]:
                for o in (s_.outs if isinstance(s_, (MultiplicityStep, TupleMultiplicityStep)) else [s_.out]):
                    step_out[o] = s_
        exposed = []  # exposed values in step order (board/logup.go:183-191)
        for rd in self.rounds:
            for s_ in rd["steps"]:
                if isinstance(s_, LogupStep):
                    exposed.append(s_.total)
                elif isinstance(s_, RunningRatioStep):
                    exposed.append(s_.end)
        exposed_idx = {nm: i for i, nm in enumerate(exposed)}
        staged: List[List[str]] = []
        seen = {}
        for r, rd in enumerate(self.rounds):
            lst = []
            for nm in rd["staged"]:
                if nm in self.setup_names:  # setup leaves are never staged (board/rounds.go:194)
                    continue
                if nm in seen:
                    raise ValueError(f"column {nm} staged twice")
                if nm not in owner:
                    raise ValueError(f"column {nm} staged at round {r} is not referenced by any relation")
                seen[nm] = r
                lst.append(nm)
            staged.append(lst)
        for nm in sorted(owner):  # sweep into the last round, sorted by name
            if nm not in seen and nm not in self.setup_names:
                seen[nm] = n_rounds - 1
                staged[-1].append(nm)

        # column table: committed columns (witness or step outputs), then the
        # Lagrange verifier columns
        def field_of(e: Expr, fields) -> int:
            if e.op == OP_COL:
                return fields.get(e.a, BASE)
            if e.op in (OP_COIN, OP_EXPAVG, OP_EXPVAL):
                return EXT
            if e.op == OP_CONST:
                return BASE
            return max(field_of(e.a, fields), field_of(e.b, fields))

        fields: Dict[str, int] = {}
        for rd in self.rounds:
            for s_ in rd["steps"]:
                if isinstance(s_, GrandProductStep):
                    fields[s_.out] = max(field_of(s_.num, fields), field_of(s_.den, fields))
                elif isinstance(s_, (LogupStep, RunningRatioStep)):
                    fields[s_.out] = EXT
                else:  # multiplicity columns
                    for o in s_.outs:
                        fields[o] = BASE
        columns: List[Tuple[str, int, int, int, int]] = []  # name, module idx, field, kind, param
        mod_names = list(self.modules)
        mod_idx = {n: i for i, n in enumerate(mod_names)}
        col_idx: Dict[str, int] = {}
        for nm in self.setup_names:
            if nm in step_out or nm in verifier:
                raise ValueError(f"setup column {nm} is a step output or a verifier column")
        for nm in sorted(owner):
            kind = KIND_STEP if nm in step_out else KIND_SETUP if nm in self.setup_names else KIND_WITNESS
            col_idx[nm] = len(columns)
            columns.append((nm, mod_idx[owner[nm]], fields.get(nm, BASE), kind, 0))
        for nm, (mname, row) in sorted(verifier.items()):
            col_idx[nm] = len(columns)
            columns.append((nm, mod_idx[mname], BASE, KIND_LAGRANGE, row))

        nodes: List[Tuple[int, int, int]] = []
        memo: Dict[tuple, int] = {}

        def emit(e: Expr) -> int:
            k = e.key()
            if k in memo:
                return memo[k]
            if e.op == OP_COL:
                if e.a not in col_idx:
                    raise ValueError(f"column {e.a} is not part of the program")
                t = (OP_COL, col_idx[e.a], e.b & 0xFFFFFFFF)
            elif e.op == OP_COIN:
                if e.a >= n_rounds:
                    raise ValueError(f"coin {e.a} beyond the {n_rounds} rounds")
                t = (OP_COIN, e.a, 0)
            elif e.op == OP_CONST:
                t = (OP_CONST, e.a, 0)
            elif e.op in (OP_EXPAVG, OP_EXPVAL):
                if e.a not in exposed_idx:
                    raise ValueError(f"exposed value {e.a} is not produced by any step")
                t = (e.op, exposed_idx[e.a], 0)
            else:
                a, b = emit(e.a), emit(e.b)
                t = (e.op, a, b)
            nodes.append(t)
            memo[k] = len(nodes) - 1
            return memo[k]

        mod_rels = [[emit(r) for r in self.modules[n].relations] for n in mod_names]
        steps = []
        for rd in self.rounds:
            for s_ in rd["steps"]:
                if isinstance(s_, GrandProductStep):
                    steps.append((STEP_GP, s_.round, mod_idx[s_.module], emit(s_.num), emit(s_.den), col_idx[s_.out]))
                elif isinstance(s_, RunningRatioStep):
                    steps.append((STEP_RATIO, s_.round, mod_idx[s_.module], emit(s_.num), emit(s_.den),
                                  col_idx[s_.out]))
                elif isinstance(s_, MultiplicityStep):
                    steps.append((STEP_MULT, s_.round, len(s_.sources), len(s_.targets),
                                  *[emit(x) for x in s_.sources], *[emit(x) for x in s_.targets],
                                  *[col_idx[o] for o in s_.outs]))
                elif isinstance(s_, TupleMultiplicityStep):
                    flags = (s_.sel_s is not None) | ((s_.sel_t is not None) << 1)
                    steps.append((STEP_MULTW, s_.round, s_.width, len(s_.sources), len(s_.targets), flags,
                                  *[emit(x) for x in (s_.sel_s or [])], *[emit(x) for x in (s_.sel_t or [])],
                                  *[emit(x) for t in s_.sources for x in t], *[emit(x) for t in s_.targets for x in t],
                                  *[col_idx[o] for o in s_.outs]))
                else:
                    w_ = [STEP_LOGUP, s_.round, mod_idx[s_.module], col_idx[s_.out], len(s_.terms)]
                    for e_, m_ in s_.terms:
                        w_ += [emit(e_), emit(m_)]
                    steps.append(tuple(w_))

        w: List[int] = [MAGIC, n_rounds, len(mod_names), len(columns), len(nodes), len(steps)]

        def wstr(s: str):
            b = s.encode()
            w.append(len(b))
            b += b"\0" * (-len(b) % 4)
            w.extend(int.from_bytes(b[i:i + 4], "little") for i in range(0, len(b), 4))

        for i, n in enumerate(mod_names):
            m = self.modules[n]
            logn = m.n.bit_length() - 1
            if m.n != 1 << logn:
                raise ValueError(f"module {n}: size {m.n} is not a power of two")
            w.append(logn)
            wstr(n)
            w.append(len(mod_rels[i]))
            w.extend(mod_rels[i])
        for (nm, mi, fld, kind, param) in columns:
            wstr(nm)
            w.extend([mi, fld, kind, param & 0xFFFFFFFF])
        for t in nodes:
            w.extend(t)
        for s in steps:
            w.extend(s)
        for lst in staged:
            w.append(len(lst))
            w.extend(col_idx[nm] for nm in lst)
        witness = [(nm, fld, self.modules[mod_names[mi]].n) for (nm, mi, fld, kind, _) in columns if kind == KIND_WITNESS]
        setup = [(nm, fld, self.modules[mod_names[mi]].n) for (nm, mi, fld, kind, _) in columns if kind == KIND_SETUP]
        return Compiled(np.array(w, dtype=np.uint32), witness, {n: self.modules[n].n for n in mod_names}, n_rounds,
                        [list(x) for x in self.logup_buses], [list(x) for x in self.product_buses], setup)


# ---------------------------------------------------------------------- arguments
def permutation_within_module(b: Builder, module: str, A: Sequence[Expr], B: Sequence[Expr]):
    """arguments/permutation.go:37-68."""
    b.stage_leaves(ROUND_FOLD, *A)
    b.stage_leaves(ROUND_FOLD, *B)
    gamma = coin(ROUND_LOG_DERIVATIVE)
    amul, bmul = A[0] - gamma, B[0] - gamma
    for x in A[1:]:
        amul = amul * (x - gamma)
    for x in B[1:]:
        bmul = bmul * (x - gamma)
    gp = b.fresh_name("gp_")
    b.add_grand_product_step(ROUND_RUNNING_SUMS, module, amul, bmul, gp)
    b.modules[module].assert_equal_at(const(1), col(gp), 0)


def logup_constraint_degree(terms: Sequence[Tuple[Expr, Expr]]) -> int:
    """board/logup.go:41-51."""
    sum_e = sum(e.degree() for e, _ in terms)
    deg = 1 + sum_e
    for e, m in terms:
        deg = max(deg, m.degree() + sum_e - e.degree())
    return deg


def range_module_name(bound: int) -> str:
    return f"{RANGE_MODULE}_{bound}"


def range_col_name(bound: int) -> str:
    return f"{RANGE_MODULE}.bound_{bound}"


def range_check(b: "Builder", S: Expr, s_module: str, bound: int):
    """arguments/lookup.go:31-47 Range: S ⊂ {0, .., bound-1} (bound rounded up
    to a power of two); the range module and its column are created on first
    use (board/module.go:56-71: values 0..bound-1 on its `bound` rows)."""
    bound = 1 << max(0, (bound - 1).bit_length())
    rm = range_module_name(bound)
    if rm not in b.modules:
        b.add_module(Module(rm, bound))
        b.generated[range_col_name(bound)] = np.arange(bound, dtype=np.uint32)
    lookup(b, [(S, s_module)], [(col(range_col_name(bound)), rm)])


def lookup(b: "Builder", S: Sequence[Tuple[Expr, str]], T: Sequence[Tuple[Expr, str]]):
    """arguments/lookup.go:53-80 LookupUnion of width-1 tables (expression,
    module): stage the tables and their multiplicities at RoundFold, then one
    cyclic logup column per module at RoundRunningSums with fractions
    1/(s - gamma) and -m/(t - gamma)."""
    mult = b.fresh_name("Mult_")
    for e, _ in list(S) + list(T):
        b.stage_leaves(ROUND_FOLD, e)
    outs = b.add_lookup_multiplicity_step(ROUND_FOLD, [e for e, _ in S], [e for e, _ in T], mult)
    b.stage_columns(ROUND_FOLD, *outs)
    gamma = coin(ROUND_LOG_DERIVATIVE)
    minus_one = const(F.P - 1)
    terms = [(mod, e - gamma, const(1)) for e, mod in S]
    terms += [(mod, e - gamma, minus_one * col(outs[i])) for i, (e, mod) in enumerate(T)]
    totals = add_logup_columns(b, f"{LOGUP}_", terms)
    b.logup_buses.append(list(totals))  # arguments/lookup.go:177
    return totals


def lookup_tuple(b: "Builder", S: Sequence[Tuple[Sequence[Expr], str]], T: Sequence[Tuple[Sequence[Expr], str]],
                 sel_s: Optional[Sequence[Expr]] = None, sel_t: Optional[Sequence[Expr]] = None):
    """arguments/lookup.go:60-110 LookupUnionTuple / CLookupUnionTuple: the
    rows of the source tables (tuples of expressions, with their module)
    whose selector is non-zero lie among the selected rows of the target
    tables.  Multiplicities are counted on the raw tuples at RoundFold; the
    logup folds each tuple with alpha = Coin(RoundFold), fractions
    sel_s/(s - gamma) and -m sel_t/(t - gamma)."""
    if sel_s is not None and len(sel_s) != len(S):
        raise ValueError("lookup: one source selector per source table")
    if sel_t is not None and len(sel_t) != len(T):
        raise ValueError("lookup: one target selector per target table")
    mult = b.fresh_name("Mult_")
    for t, _ in list(S) + list(T):
        b.stage_leaves(ROUND_FOLD, *t)
    b.stage_leaves(ROUND_FOLD, *(sel_s or []))
    b.stage_leaves(ROUND_FOLD, *(sel_t or []))
    outs = b.add_tuple_multiplicity_step(ROUND_FOLD, sel_s, sel_t, [t for t, _ in S], [t for t, _ in T], mult)
    b.stage_columns(ROUND_FOLD, *outs)
    alpha, gamma, minus_one = coin(ROUND_FOLD), coin(ROUND_LOG_DERIVATIVE), const(F.P - 1)

    def folded(t):  # arguments/lookup.go:232-244
        return t[0] if len(t) == 1 else fold(alpha, list(t))

    terms = [(mod, folded(t) - gamma, const(1) if sel_s is None else sel_s[i]) for i, (t, mod) in enumerate(S)]
    terms += [(mod, folded(t) - gamma, minus_one * (col(outs[i]) if sel_t is None else col(outs[i]) * sel_t[i]))
              for i, (t, mod) in enumerate(T)]
    totals = add_logup_columns(b, f"{LOGUP}_", terms)
    b.logup_buses.append(list(totals))
    return totals


def running_ratio_constraint_degree(num: Sequence[Expr], den: Sequence[Expr]) -> int:
    """board/product.go:43-52."""
    return max(1 + sum(f.degree() for f in num), 2 + sum(f.degree() for f in den))


def bus(b: "Builder", sel_s: Sequence[Expr], sel_r: Sequence[Expr], S: Sequence[Tuple[Sequence[Expr], str]],
        R: Sequence[Tuple[Sequence[Expr], str]]) -> List[str]:
    """arguments/bus.go:42-67 Bus: the tuples S[i] (sent on the rows where
    sel_s[i] = 1) and R[i] (received where sel_r[i] = 1) balance as
    multisets.  Tables are (expressions of the tuple, module).  Every selected
    row contributes the factor beta + alpha^w + alpha^(w-1) c_(w-1) + ... + c_0
    (sends as numerators, receives as denominators) and an unselected row 1,
    as sel (factor - 1) + 1; the factors go into running-ratio columns whose
    ends form a product bus.  Returns the ends."""
    if len(sel_s) != len(S) or len(sel_r) != len(R):
        raise ValueError("bus: one selector per table")
    if not S and not R:
        return []
    tables = list(S) + list(R)
    if len({len(t) for t, _ in tables}) != 1:
        raise ValueError("bus: inconsistent width")
    for t, _ in tables:
        b.stage_leaves(ROUND_FOLD, *t)
    b.stage_leaves(ROUND_FOLD, *sel_s)
    b.stage_leaves(ROUND_FOLD, *sel_r)
    ends = _add_running_ratios(b, _bus_factors(S, sel_s), _bus_factors(R, sel_r))
    b.product_buses.append(list(ends))  # arguments/bus.go:66
    return ends


def _bus_factors(tables, sels) -> List[Tuple[str, Expr]]:
    """arguments/bus.go:76-90: sel (beta + fold(row) - 1) + 1, fold by Horner
    from the sentinel alpha^w."""
    alpha, beta, one = coin(ROUND_FOLD), coin(ROUND_LOG_DERIVATIVE), const(1)
    res = []
    for (t, module), sel in zip(tables, sels):
        f = alpha + t[-1]
        for c in reversed(t[:-1]):
            f = f * alpha + c
        res.append((module, sel * (f + beta - one) + one))
    return res


def _add_running_ratios(b: "Builder", num, den) -> List[str]:
    """arguments/bus.go:98-137: factors grouped by module (first-appearance
    order) into running-ratio columns at RoundRunningSums, each taking in turn
    the module's next denominator and next numerator while the constraint
    degree stays within MAX_LOGUP_DEGREE."""
    order: List[str] = []
    by_mod: Dict[str, Tuple[List[Expr], List[Expr]]] = {}
    for side, fs in ((0, num), (1, den)):
        for module, f in fs:
            if module not in by_mod:
                order.append(module)
                by_mod[module] = ([], [])
            by_mod[module][side].append(f)
    ends = []
    for module in order:
        nums, dens = list(by_mod[module][0]), list(by_mod[module][1])
        while nums or dens:
            cn: List[Expr] = []
            cd: List[Expr] = []
            grown = True
            while grown:
                grown = False
                if dens and running_ratio_constraint_degree(cn, cd + [dens[0]]) <= MAX_LOGUP_DEGREE:
                    cd.append(dens.pop(0))
                    grown = True
                if nums and running_ratio_constraint_degree(cn + [nums[0]], cd) <= MAX_LOGUP_DEGREE:
                    cn.append(nums.pop(0))
                    grown = True
            if not cn and not cd:
                raise ValueError(f"module {module}: a bus factor alone exceeds degree {MAX_LOGUP_DEGREE}")
            ends.append(b.add_running_ratio_step(ROUND_RUNNING_SUMS, module, cn, cd, b.fresh_name(f"{module}.busratio_")))
    return ends


def add_logup_columns(b: "Builder", prefix: str, terms: Sequence[Tuple[str, Expr, Expr]]) -> List[str]:
    """arguments/lookup.go:176-214: terms grouped by module (first-appearance
    order), batched up to MAX_LOGUP_BATCH per column within the degree bound."""
    order: List[str] = []
    by_mod: Dict[str, List[Tuple[Expr, Expr]]] = {}
    for mod, e, m in terms:
        if mod not in by_mod:
            order.append(mod)
            by_mod[mod] = []
        by_mod[mod].append((e, m))
    totals = []
    for mod in order:
        ts = by_mod[mod]
        while ts:
            n = 1
            while n < min(MAX_LOGUP_BATCH, len(ts)) and logup_constraint_degree(ts[:n + 1]) <= MAX_LOGUP_DEGREE:
                n += 1
            name = b.fresh_name(f"{mod}.{prefix}") + "_0"
            totals.append(b.add_cyclic_logup_step(ROUND_RUNNING_SUMS, mod, ts[:n], name))
            ts = ts[n:]
    return totals


def id_support(n_chunks: int, n: int) -> List[np.ndarray]:
    """ID_k[j] = g^k w^j, g = 3 (board/module.go:262-281); canonical values."""
    w = F.root_of_unity(n)
    res = [F.powers(w, n)]
    for _ in range(1, n_chunks):
        res.append(((res[-1].astype(np.uint64) * F.MULT_GEN) % F.P).astype(np.uint32))
    return res


def copy_constraint(b: Builder, module: str, A: Sequence[Expr], S: np.ndarray, perm_name: str):
    """arguments/permutation.go:101-127 with board.PermutationGen: sigma_k[j] is
    the ID-support value at position S[k*N + j]."""
    m = b.modules[module]
    n = m.n
    if len(S) != n * len(A):
        raise ValueError("len(S) must equal N * len(A)")
    sup = id_support(len(A), n)
    flat = np.concatenate(sup)
    alpha = coin(ROUND_FOLD)
    fa, fb = [], []
    for i, a in enumerate(A):
        idn = m.id_support_name(i)
        sgn = f"{perm_name}_{i}"
        b.generated[idn] = sup[i]
        b.generated[sgn] = flat[np.asarray(S[i * n:(i + 1) * n], dtype=np.int64)]
        fa.append(fold(alpha, [a, col(idn)]))
        fb.append(fold(alpha, [a, col(sgn)]))
    permutation_within_module(b, module, fa, fb)
