// CPU oracle (test infrastructure): the prover's state and its phases, shared
// by the prove flow (oracle_prover.cpp) and the verifier
// (oracle_verifier.cpp), which reuses the program layout: relation folding,
// degrees, shift schedule, tree layout and chunk counts.  Reference flow:
// prover/prover.go:142-719; layout internal/protocol/layout.go:107-247;
// schedule internal/protocol/schedule.go:92-235.
#pragma once
#include <algorithm>
#include <cstring>
#include <map>
#include <set>
#include <stdexcept>

#include "oracle.h"
#include "program.h"

namespace orc {

namespace {

const uint64_t RATE = 4;
const int MAX_LOG = 22;
const uint64_t N_FRI = RATE << MAX_LOG;

std::string coin_name(int r) { return "challenge@loom_" + std::to_string(r); }

// ------------------------------------------------------------ serialization
struct Writer {
  std::vector<uint8_t> b;
  void u32(uint32_t x) { for (int i = 3; i >= 0; i--) b.push_back((uint8_t)(x >> (8 * i))); }
  void el(uint32_t x) { u32(x); }
  void e6(const E6& x) { for (int i = 0; i < 6; i++) el(x.c[i]); }
  void dg(const Digest& d) { for (int i = 0; i < 8; i++) el(d.v[i]); }
  void str(const std::string& s) { u32((uint32_t)s.size()); b.insert(b.end(), s.begin(), s.end()); }
};

// ------------------------------------------------------------ expressions
struct Val { bool ext; uint32_t b; E6 e; };
inline E6 as_e6(const Val& v) { return v.ext ? v.e : e6_from_base(v.b); }
inline Val vb(uint32_t x) { Val v; v.ext = false; v.b = x; return v; }
inline Val ve(const E6& x) { Val v; v.ext = true; v.e = x; v.b = 0; return v; }
Val vadd(const Val& x, const Val& y) { if (!x.ext && !y.ext) return vb(add(x.b, y.b)); return ve(e6_add(as_e6(x), as_e6(y))); }
Val vsub(const Val& x, const Val& y) { if (!x.ext && !y.ext) return vb(sub(x.b, y.b)); return ve(e6_sub(as_e6(x), as_e6(y))); }
Val vmul(const Val& x, const Val& y) {
  if (!x.ext && !y.ext) return vb(mul(x.b, y.b));
  if (!x.ext) return ve(e6_mul_base(y.e, x.b));
  if (!y.ext) return ve(e6_mul_base(x.e, y.b));
  return ve(e6_mul(x.e, y.e));
}

const int NEG_INF = -1000000;
inline bool is_binary(uint32_t op) { return op == OP_ADD || op == OP_SUB || op == OP_MUL; }

struct Prover {
  const Program& pg;
  uint32_t num_queries;
  Transcript fs;
  std::vector<E6> coins;              // per round
  std::vector<E6> exposed;            // logup totals, in step order
  std::vector<std::string> exposed_names;
  std::map<uint32_t, std::vector<uint32_t>> base;  // column id -> Lagrange-normal values
  std::map<uint32_t, std::vector<E6>> ext;
  std::vector<uint32_t> mod_order;    // module ids sorted by name

  // Folded vanishing relation per module: extra nodes appended to a copy.
  std::vector<PNode> nodes;
  std::vector<int> fold_root;         // per module, -1 when no relation
  std::vector<int> degree;            // per module
  std::vector<bool> root_ext;

  // Layout: trees in canonical order (rounds with staged columns, then AIR).
  struct Group { uint32_t module; std::vector<uint32_t> bcols, ecols; };  // column ids, or chunk ids for AIR
  struct TreeL { bool air; int round; std::vector<Group> groups; bool setup = false; };
  std::vector<TreeL> trees;
  // AIR chunks: (module, chunk) -> Lagrange-normal polynomial.
  std::map<std::pair<uint32_t, uint32_t>, std::vector<uint32_t>> air_base;
  std::map<std::pair<uint32_t, uint32_t>, std::vector<E6>> air_ext;
  std::map<uint32_t, std::vector<int>> col_shifts;  // committed column -> sorted normalized shifts

  struct Source { std::vector<std::vector<uint32_t>> b; std::vector<std::vector<E6>> e; size_t rows; };
  struct Committed { Tree tree; std::vector<Source> sources; };  // sources in sorted order
  std::vector<Committed> committed;
  std::vector<Digest> commitments;   // trace and AIR roots (the proof's)
  Digest setup_root{};               // the verification key when there is a setup tree
  E6 zeta;

  Prover(const Program& p, uint32_t q) : pg(p), num_queries(q) {}

  size_t mod_n(uint32_t m) const { return (size_t)1 << pg.modules[m].log_n; }

  // ---------------------------------------------------------- node helpers
  uint32_t push(uint32_t op, uint32_t a, uint32_t b) { nodes.push_back({op, a, b}); return (uint32_t)nodes.size() - 1; }
  int node_degree(uint32_t id, std::vector<int>& memo) {
    if (memo[id] != INT32_MIN) return memo[id];
    const PNode& x = nodes[id];
    int d = 0;
    switch (x.op) {
      case OP_COL: d = 1; break;
      case OP_EXPAVG: d = 1; break;  // a verifier column (internal/dag/dag.go:1536)
      case OP_EXPVAL: d = 0; break;  // a constant (times L_0 it is the sparse column)
      case OP_COIN: d = 0; break;
      case OP_CONST: d = x.a == 0 ? NEG_INF : 0; break;
      case OP_ADD: case OP_SUB: d = std::max(node_degree(x.a, memo), node_degree(x.b, memo)); break;
      case OP_MUL: {
        int l = node_degree(x.a, memo), r = node_degree(x.b, memo);
        d = (l == NEG_INF || r == NEG_INF) ? NEG_INF : l + r;
        break;
      }
    }
    return memo[id] = d;
  }
  bool node_ext(uint32_t id, std::vector<int>& memo) {
    if (memo[id] >= 0) return memo[id];
    const PNode& x = nodes[id];
    bool e = false;
    if (x.op == OP_COL) e = pg.columns[x.a].field == 1;
    else if (x.op == OP_COIN || x.op == OP_EXPAVG || x.op == OP_EXPVAL) e = true;
    else if (is_binary(x.op)) e = node_ext(x.a, memo) || node_ext(x.b, memo);
    memo[id] = e;
    return e;
  }
  void collect(uint32_t id, std::vector<char>& seen, std::vector<uint32_t>& order) {
    if (seen[id]) return;
    seen[id] = 1;
    const PNode& x = nodes[id];
    if (is_binary(x.op)) { collect(x.a, seen, order); collect(x.b, seen, order); }
    order.push_back(id);
  }

  // Evaluate `root` at row j of a size-n vector family. colval(col, row)
  // returns the value of column col at the (shift-adjusted) row.
  template <class F> Val eval(const std::vector<uint32_t>& order, uint32_t root, size_t j, size_t n, F colval, std::vector<Val>& scratch) {
    for (uint32_t id : order) {
      const PNode& x = nodes[id];
      Val v;
      switch (x.op) {
        case OP_COL: {
          int64_t sh = (int32_t)x.b;
          size_t r = (size_t)((((int64_t)j + sh) % (int64_t)n + (int64_t)n) % (int64_t)n);
          v = colval(x.a, r);
          break;
        }
        case OP_COIN: v = ve(coins.at(x.a)); break;
        case OP_CONST: v = vb(x.a); break;
        case OP_EXPAVG: v = ve(e6_mul_base(exposed.at(x.a), inv((uint32_t)n))); break;
        case OP_EXPVAL: v = ve(exposed.at(x.a)); break;
        case OP_ADD: v = vadd(scratch[x.a], scratch[x.b]); break;
        case OP_SUB: v = vsub(scratch[x.a], scratch[x.b]); break;
        default: v = vmul(scratch[x.a], scratch[x.b]); break;
      }
      scratch[id] = v;
    }
    return scratch[root];
  }

  // ---------------------------------------------------------- setup
  void setup(const uint32_t* const* witness) {
    setup_layout();
    load_columns(witness);
  }
  // values of column c from Montgomery words
  void load_column(uint32_t c, const uint32_t* src) {
    size_t n = mod_n(pg.columns[c].module);
    if (pg.columns[c].field == 0) {
      std::vector<uint32_t> v(n);
      for (size_t i = 0; i < n; i++) v[i] = from_mont(src[i]);
      base[c] = v;
    } else {
      std::vector<E6> v(n);
      for (size_t i = 0; i < n; i++) for (int k = 0; k < 6; k++) v[i].c[k] = from_mont(src[6 * i + k]);
      ext[c] = v;
    }
  }
  // The setup tree's root (the verification key) from the setup columns
  // alone, in descriptor order (setup/setup.go:68-124).
  Digest setup_commit(const uint32_t* const* setup) {
    setup_layout();
    size_t si = 0;
    for (uint32_t c = 0; c < pg.columns.size(); c++)
      if (pg.columns[c].kind == KIND_SETUP) load_column(c, setup[si++]);
    if (trees.empty() || !trees[0].setup) throw std::runtime_error("setup: the program has no setup columns");
    return commit(tree_groups(trees[0])).tree.root();
  }
  // witness columns, then setup columns (each in descriptor order, as
  // `witness` lists them), and the Lagrange columns' values
  void load_columns(const uint32_t* const* witness) {
    size_t nw = 0;
    for (const PColumn& col : pg.columns) nw += col.kind == KIND_WITNESS;
    size_t wi = 0, si = nw;
    for (uint32_t c = 0; c < pg.columns.size(); c++) {
      const PColumn& col = pg.columns[c];
      size_t n = mod_n(col.module);
      if (col.kind == KIND_WITNESS || col.kind == KIND_SETUP) {
        load_column(c, witness[col.kind == KIND_WITNESS ? wi++ : si++]);
      } else if (col.kind == KIND_LAGRANGE) {
        // board/module.go:56-82: 1 at row i (or N-1-i for relative columns)
        std::vector<uint32_t> v(n, 0);
        int64_t row = col.param >= 0 ? col.param : (int64_t)n - 1 - (-(int64_t)col.param - 1);
        if (row < 0 || row >= (int64_t)n) throw std::runtime_error("Lagrange column row out of range");
        v[row] = 1;
        base[c] = v;
      }
    }
  }
  // Everything the verifier shares: module order, folded relations, degrees,
  // shift schedule and tree layout (no witness needed).
  void setup_layout() {
    nodes = pg.nodes;
    // module order: sort.Strings on names (internal/protocol/layout.go:107-114)
    for (uint32_t m = 0; m < pg.modules.size(); m++) mod_order.push_back(m);
    std::sort(mod_order.begin(), mod_order.end(), [&](uint32_t a, uint32_t b) { return pg.modules[a].name < pg.modules[b].name; });
    // fold relations: C0 + c(C1 + c(C2 + ...)), c = coin(last round)
    // (board/program.go:62-80, expr/utils.go:21-33)
    fold_root.assign(pg.modules.size(), -1);
    degree.assign(pg.modules.size(), NEG_INF);
    root_ext.assign(pg.modules.size(), false);
    for (uint32_t m = 0; m < pg.modules.size(); m++) {
      const auto& rels = pg.modules[m].rels;
      if (rels.empty()) continue;
      uint32_t res = rels.back();
      for (int i = (int)rels.size() - 2; i >= 0; i--) {
        uint32_t c = push(OP_COIN, pg.n_rounds - 1, 0);
        uint32_t t = push(OP_MUL, c, res);
        res = push(OP_ADD, rels[i], t);
      }
      fold_root[m] = (int)res;
    }
    for (uint32_t m = 0; m < pg.modules.size(); m++) {
      if (fold_root[m] < 0) continue;
      std::vector<int> dm(nodes.size(), INT32_MIN), em(nodes.size(), -1);
      degree[m] = node_degree(fold_root[m], dm);
      root_ext[m] = node_ext(fold_root[m], em);
    }
    // shift schedule: normalized shifts of committed leaves in the folded
    // relations (internal/protocol/schedule.go:92-157)
    for (uint32_t m : mod_order) {
      if (fold_root[m] < 0) continue;
      std::vector<char> seen(nodes.size(), 0);
      std::vector<uint32_t> order;
      collect(fold_root[m], seen, order);
      int64_t n = (int64_t)mod_n(m);
      for (uint32_t id : order) {
        if (nodes[id].op != OP_COL) continue;
        const PColumn& col = pg.columns[nodes[id].a];
        if (col.kind == KIND_LAGRANGE) continue;  // verifier column
        int64_t sh = (int32_t)nodes[id].b;
        int s = (int)(((sh % n) + n) % n);
        auto& v = col_shifts[nodes[id].a];
        if (std::find(v.begin(), v.end(), s) == v.end()) v.push_back(s);
      }
    }
    for (auto& kv : col_shifts) std::sort(kv.second.begin(), kv.second.end());
    // layout (internal/protocol/layout.go:165-241): the setup tree (setup
    // columns by module, sorted by name within a module, base then ext;
    // internal/protocol/layout.go:131-151), one tree per round with staged
    // columns, then one AIR tree; groups in sorted module order.
    {
      TreeL t; t.air = false; t.round = -2; t.setup = true;
      for (uint32_t m : mod_order) {
        std::vector<uint32_t> cols;
        for (uint32_t c = 0; c < pg.columns.size(); c++)
          if (pg.columns[c].kind == KIND_SETUP && pg.columns[c].module == m) cols.push_back(c);
        std::sort(cols.begin(), cols.end(), [&](uint32_t a, uint32_t b) { return pg.columns[a].name < pg.columns[b].name; });
        Group g; g.module = m;
        for (uint32_t c : cols) (pg.columns[c].field == 0 ? g.bcols : g.ecols).push_back(c);
        if (!g.bcols.empty() || !g.ecols.empty()) t.groups.push_back(g);
      }
      if (!t.groups.empty()) trees.push_back(t);
    }
    for (uint32_t r = 0; r < pg.n_rounds; r++) {
      TreeL t; t.air = false; t.round = (int)r;
      for (uint32_t m : mod_order) {
        Group g; g.module = m;
        for (uint32_t c : pg.staged[r]) {
          if (pg.columns[c].module != m) continue;
          (pg.columns[c].field == 0 ? g.bcols : g.ecols).push_back(c);
        }
        if (!g.bcols.empty() || !g.ecols.empty()) t.groups.push_back(g);
      }
      if (!t.groups.empty()) trees.push_back(t);
    }
    {
      TreeL t; t.air = true; t.round = -1;
      for (uint32_t m : mod_order) {
        uint32_t nch = chunk_count(m);
        if (!nch) continue;
        Group g; g.module = m;
        for (uint32_t k = 0; k < nch; k++) (root_ext[m] ? g.ecols : g.bcols).push_back(k);
        t.groups.push_back(g);
      }
      if (!t.groups.empty()) trees.push_back(t);
    }
  }

  // internal/poly/compute_quotient.go:508-510, internal/protocol/layout.go:155-160
  uint32_t chunk_count(uint32_t m) const {
    if (fold_root[m] < 0 || degree[m] <= 0) return 0;
    size_t n = mod_n(m);
    size_t want = (size_t)std::max(degree[m] - 1, 1) * n, big = 1;
    while (big < want) big <<= 1;
    return (uint32_t)(big / n);
  }

  // ---------------------------------------------------------- commit
  struct GroupData { std::vector<const uint32_t*> b; std::vector<const E6*> e; size_t n; };
  Committed commit(const std::vector<GroupData>& groups) {
    std::vector<size_t> order(groups.size());
    for (size_t i = 0; i < order.size(); i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return groups[a].n > groups[b].n; });
    Committed c;
    std::vector<std::vector<Digest>> leaves;
    // every column of every group is encoded independently: one parallel
    // loop over all of them (the reference fans out per column,
    // internal/fri/commitment.go:303-331)
    c.sources.resize(order.size());
    struct Job { size_t k, i; bool ext; };
    std::vector<Job> jobs;
    for (size_t k = 0; k < order.size(); k++) {
      const GroupData& g = groups[order[k]];
      Source& s = c.sources[k];
      s.rows = RATE * g.n;
      s.b.resize(g.b.size());
      s.e.resize(g.e.size());
      for (size_t i = 0; i < g.b.size(); i++) jobs.push_back({k, i, false});
      for (size_t i = 0; i < g.e.size(); i++) jobs.push_back({k, i, true});
    }
#pragma omp parallel for schedule(dynamic)
    for (size_t q = 0; q < jobs.size(); q++) {
      const Job& jb = jobs[q];
      const GroupData& g = groups[order[jb.k]];
      Source& s = c.sources[jb.k];
      if (jb.ext) s.e[jb.i] = rs_encode_e6(g.e[jb.i], g.n, s.rows);
      else s.b[jb.i] = rs_encode(g.b[jb.i], g.n, s.rows);
    }
    for (size_t k = 0; k < order.size(); k++) leaves.push_back(hash_leaf_pairs(c.sources[k]));
    std::vector<Injection> inj;
    for (size_t k = 1; k < leaves.size(); k++) inj.push_back(Injection{leaves[k]});
    c.tree = build_tree(leaves[0], inj);
    return c;
  }
  // leaf k = Sponge(LEAF, 2nB, 2nE, lo.base, hi.base, lo.ext, hi.ext)
  // (internal/fri/hash.go:39-57)
  static std::vector<Digest> hash_leaf_pairs(const Source& s) {
    std::vector<Digest> out(s.rows / 2);
#pragma omp parallel for schedule(static)
    for (size_t k = 0; k < s.rows / 2; k++) {
      Sponge h;
      h.write((uint32_t)LEAF_TAG);
      h.write((uint32_t)(2 * s.b.size()));
      h.write((uint32_t)(2 * s.e.size()));
      for (auto& col : s.b) h.write(col[2 * k]);
      for (auto& col : s.b) h.write(col[2 * k + 1]);
      for (auto& col : s.e) h.write_e6(col[2 * k]);
      for (auto& col : s.e) h.write_e6(col[2 * k + 1]);
      out[k] = h.sum();
    }
    return out;
  }
  std::vector<GroupData> tree_groups(const TreeL& t) {
    std::vector<GroupData> gs;
    for (const Group& g : t.groups) {
      GroupData d; d.n = mod_n(g.module);
      for (uint32_t c : g.bcols) d.b.push_back(t.air ? air_base.at({g.module, c}).data() : base.at(c).data());
      for (uint32_t c : g.ecols) d.e.push_back(t.air ? air_ext.at({g.module, c}).data() : ext.at(c).data());
      gs.push_back(d);
    }
    return gs;
  }

  // ---------------------------------------------------------- steps
  // Grand product R[0] = 1, R[i+1] = R[i] num(i)/den(i)
  // (internal/poly/iop_utils.go:170-192,316-323)
  // module whose rows an expression ranges over: that of its first column
  uint32_t expr_module(uint32_t root) {
    std::vector<char> seen(nodes.size(), 0);
    std::vector<uint32_t> order;
    collect(root, seen, order);
    for (uint32_t id : order)
      if (nodes[id].op == OP_COL) return pg.columns[nodes[id].a].module;
    throw std::runtime_error("lookup table without a column");
  }
  std::vector<uint32_t> eval_base_rows(uint32_t root, uint32_t module) {
    size_t n = mod_n(module);
    std::vector<char> seen(nodes.size(), 0);
    std::vector<uint32_t> order;
    collect(root, seen, order);
    auto colval = [&](uint32_t c, size_t r) -> Val {
      if (pg.columns[c].field == 0) return vb(base.at(c)[r]);
      return ve(ext.at(c)[r]);
    };
    std::vector<uint32_t> out(n);
    std::vector<Val> sc(nodes.size());
    for (size_t j = 0; j < n; j++) {
      Val v = eval(order, root, j, n, colval, sc);
      if (v.ext) throw std::runtime_error("lookup table values must be base-field");
      out[j] = v.b;
    }
    return out;
  }

  // Lookup multiplicities of width-1 tables (internal/poly/lookup_multiplicity.go:37-100):
  // the weight of every source value goes to its first target row (T[0]
  // rows, then T[1] rows, ...); a source value found in no target is an error.
  void run_multiplicities(const PStep& st) {
    std::map<uint32_t, uint32_t> weight;
    for (uint32_t s : st.src)
      for (uint32_t v : eval_base_rows(s, expr_module(s))) weight[v] = add(weight[v], 1);
    std::set<uint32_t> assigned;
    for (size_t k = 0; k < st.tgt.size(); k++) {
      uint32_t mod = expr_module(st.tgt[k]);
      std::vector<uint32_t> tv = eval_base_rows(st.tgt[k], mod), res(tv.size(), 0);
      for (size_t i = 0; i < tv.size(); i++) {
        auto it = weight.find(tv[i]);
        if (it == weight.end() || assigned.count(tv[i])) continue;
        res[i] = it->second;
        assigned.insert(tv[i]);
      }
      if (pg.columns[st.outs[k]].module != mod) throw std::runtime_error("multiplicity column module");
      base[st.outs[k]] = res;
    }
    for (auto& kv : weight)
      if (!assigned.count(kv.first) && kv.second) throw std::runtime_error("lookup: source value not in the table");
  }

  // Lookup multiplicities of tuples with selectors
  // (internal/poly/lookup_multiplicity.go:37-100): the selected weight of
  // every source tuple (compared on its base-field values) goes to its first
  // target row with a non-zero selector, divided by that selector; a
  // selected source tuple found in no target is an error.
  void run_multiplicities_tuple(const PStep& st) {
    const uint32_t W = st.width;
    auto table = [&](const std::vector<uint32_t>& nodes_, size_t k, std::vector<std::vector<uint32_t>>& cols) {
      uint32_t mod = expr_module(nodes_[k * W]);
      cols.clear();
      for (uint32_t w = 0; w < W; w++) {
        if (expr_module(nodes_[k * W + w]) != mod) throw std::runtime_error("lookup: a tuple spans modules");
        cols.push_back(eval_base_rows(nodes_[k * W + w], mod));
      }
      return mod;
    };
    auto selector = [&](const std::vector<uint32_t>& sels, size_t k, uint32_t mod) {
      if (sels.empty()) return std::vector<uint32_t>(mod_n(mod), 1);
      if (expr_module(sels[k]) != mod) throw std::runtime_error("lookup: selector of another module");
      return eval_base_rows(sels[k], mod);
    };
    std::map<std::vector<uint32_t>, uint32_t> weight;
    std::vector<std::vector<uint32_t>> cols;
    for (size_t k = 0; k < st.src.size() / W; k++) {
      uint32_t mod = table(st.src, k, cols);
      std::vector<uint32_t> sel = selector(st.sel_s, k, mod);
      for (size_t i = 0; i < sel.size(); i++) {
        if (!sel[i]) continue;
        std::vector<uint32_t> key(W);
        for (uint32_t w = 0; w < W; w++) key[w] = cols[w][i];
        weight[key] = add(weight[key], sel[i]);
      }
    }
    std::set<std::vector<uint32_t>> assigned;
    for (size_t k = 0; k < st.outs.size(); k++) {
      uint32_t mod = table(st.tgt, k, cols);
      std::vector<uint32_t> sel = selector(st.sel_t, k, mod), res(sel.size(), 0);
      for (size_t i = 0; i < sel.size(); i++) {
        if (!sel[i]) continue;
        std::vector<uint32_t> key(W);
        for (uint32_t w = 0; w < W; w++) key[w] = cols[w][i];
        auto it = weight.find(key);
        if (it == weight.end() || assigned.count(key)) continue;
        res[i] = mul(it->second, inv(sel[i]));
        assigned.insert(key);
      }
      if (pg.columns[st.outs[k]].module != mod || pg.columns[st.outs[k]].field != 0)
        throw std::runtime_error("multiplicity column must be a base column of its table's module");
      base[st.outs[k]] = res;
    }
    for (auto& kv : weight)
      if (kv.second && !assigned.count(kv.first)) throw std::runtime_error("lookup: source value not in the table");
  }

  // Cyclic logup column (board/logup.go:129-180, internal/poly/iop_utils.go:110-131):
  // v_i = sum_j M_j(i) / E_j(i); S_i = v_0 + ... + v_i; T = S_{n-1};
  // L_i = S_i - (i + 1) T / n.  T is exposed.
  void run_logup(const PStep& st) {
    size_t n = mod_n(st.module);
    auto colval = [&](uint32_t c, size_t r) -> Val {
      if (pg.columns[c].field == 0) return vb(base.at(c)[r]);
      return ve(ext.at(c)[r]);
    };
    std::vector<std::vector<uint32_t>> oe(st.e.size()), om(st.e.size());
    for (size_t k = 0; k < st.e.size(); k++) {
      std::vector<char> s1(nodes.size(), 0), s2(nodes.size(), 0);
      collect(st.e[k], s1, oe[k]);
      collect(st.m[k], s2, om[k]);
    }
    std::vector<E6> col(n);
    std::vector<Val> sc(nodes.size());
    E6 run = e6_zero();
    std::vector<E6> sums(n);
    for (size_t j = 0; j < n; j++) {
      E6 v = e6_zero();
      for (size_t k = 0; k < st.e.size(); k++) {
        E6 e = as_e6(eval(oe[k], st.e[k], j, n, colval, sc));
        E6 m = as_e6(eval(om[k], st.m[k], j, n, colval, sc));
        if (e6_is_zero(e)) throw std::runtime_error("logup: zero denominator");
        v = e6_add(v, e6_mul(m, e6_inv(e)));
      }
      run = e6_add(run, v);
      sums[j] = run;
    }
    E6 total = sums[n - 1];
    E6 avg = e6_mul_base(total, inv((uint32_t)n));
    E6 shift = e6_zero();
    for (size_t i = 0; i < n; i++) {
      shift = e6_add(shift, avg);
      col[i] = e6_sub(sums[i], shift);
    }
    if (pg.columns[st.out].module != st.module || pg.columns[st.out].field != 1)
      throw std::runtime_error("logup column must be an extension column of its module");
    ext[st.out] = col;
    if (exposed.size() <= st.exposed) { exposed.resize(st.exposed + 1); exposed_names.resize(st.exposed + 1); }
    exposed[st.exposed] = total;
    exposed_names[st.exposed] = pg.columns[st.out].name + "_total";
  }

  // Running ratio (board/product.go:123-198): Z_i = prod_{k<=i} num_k / den_k,
  // end P = Z_{N-1} exposed.
  void run_ratio(const PStep& st) {
    size_t n = mod_n(st.module);
    std::vector<uint32_t> order_n, order_d;
    { std::vector<char> seen(nodes.size(), 0); collect(st.num, seen, order_n); }
    { std::vector<char> seen(nodes.size(), 0); collect(st.den, seen, order_d); }
    auto colval = [&](uint32_t c, size_t r) -> Val {
      if (pg.columns[c].field == 0) return vb(base.at(c)[r]);
      return ve(ext.at(c)[r]);
    };
    std::vector<Val> sc(nodes.size());
    std::vector<E6> col(n);
    E6 acc = e6_one();
    for (size_t j = 0; j < n; j++) {
      E6 a = as_e6(eval(order_n, st.num, j, n, colval, sc));
      E6 b = as_e6(eval(order_d, st.den, j, n, colval, sc));
      if (e6_is_zero(b)) throw std::runtime_error("running ratio: zero denominator");
      acc = e6_mul(acc, e6_mul(a, e6_inv(b)));
      col[j] = acc;
    }
    if (pg.columns[st.out].module != st.module || pg.columns[st.out].field != 1)
      throw std::runtime_error("running ratio column must be an extension column of its module");
    ext[st.out] = col;
    if (exposed.size() <= st.exposed) { exposed.resize(st.exposed + 1); exposed_names.resize(st.exposed + 1); }
    exposed[st.exposed] = col[n - 1];
    exposed_names[st.exposed] = pg.columns[st.out].name + "_end";
  }

  void run_step(const PStep& st) {
    if (st.type == STEP_MULT) return run_multiplicities(st);
    if (st.type == STEP_MULTW) return run_multiplicities_tuple(st);
    if (st.type == STEP_LOGUP) return run_logup(st);
    if (st.type == STEP_RATIO) return run_ratio(st);
    if (st.type != STEP_GP) throw std::runtime_error("unsupported step type");
    size_t n = mod_n(st.module);
    std::vector<uint32_t> order_n, order_d;
    { std::vector<char> seen(nodes.size(), 0); collect(st.num, seen, order_n); }
    { std::vector<char> seen(nodes.size(), 0); collect(st.den, seen, order_d); }
    std::vector<E6> ratio(n);
    auto colval = [&](uint32_t c, size_t r) -> Val {
      if (pg.columns[c].field == 0) return vb(base.at(c)[r]);
      return ve(ext.at(c)[r]);
    };
#pragma omp parallel for schedule(static)
    for (size_t j = 0; j < n; j++) {
      std::vector<Val> sc(nodes.size());
      E6 a = as_e6(eval(order_n, st.num, j, n, colval, sc));
      E6 b = as_e6(eval(order_d, st.den, j, n, colval, sc));
      if (e6_is_zero(b)) throw std::runtime_error("grand product: zero denominator");
      ratio[j] = e6_mul(a, e6_inv(b));
    }
    std::vector<E6> r(n);
    r[0] = e6_one();
    for (size_t i = 1; i < n; i++) r[i] = e6_mul(r[i - 1], ratio[i - 1]);
    ext[st.out] = r;
  }

  // ---------------------------------------------------------- quotient
  // Q = V / (X^N - 1) evaluated on g<w_big> as rho cosets of size N, then
  // coset-Lagrange -> canonical (iFFT, x g^-k), chunked, FFT_DIF+BitReverse
  // (internal/poly/compute_quotient.go:223-424,484-499; prover/prover.go:422-440).
  // Returns the rho chunk columns (E6; base-field relations keep only
  // coordinate 0 when stored).
  std::vector<std::vector<E6>> quotient(uint32_t m) {
    size_t n = mod_n(m);
    uint32_t rho = chunk_count(m);
    size_t big = rho * n;
    std::vector<char> seen(nodes.size(), 0);
    std::vector<uint32_t> order;
    collect(fold_root[m], seen, order);
    std::set<uint32_t> cols;
    for (uint32_t id : order) if (nodes[id].op == OP_COL) cols.insert(nodes[id].a);
    // canonical coefficients of every column used
    std::map<uint32_t, std::vector<uint32_t>> cb;
    std::map<uint32_t, std::vector<E6>> ce;
    for (uint32_t c : cols) {
      if (pg.columns[c].field == 0) {
        std::vector<uint32_t> v = base.at(c);
        ifft_dif(v.data(), n); bit_reverse(v.data(), n);
        cb[c] = v;
      } else {
        std::vector<E6> v = ext.at(c);
        ifft_dif_e6(v.data(), n); bit_reverse_e6(v.data(), n);
        ce[c] = v;
      }
    }
    uint32_t g = MULT_GEN, wbig = root_of_unity(big);
    std::vector<E6> num(big);
    for (uint32_t i = 0; i < rho; i++) {
      uint32_t s = mul(g, pow(wbig, i));  // coset shift
      std::map<uint32_t, std::vector<uint32_t>> vb_;
      std::map<uint32_t, std::vector<E6>> ve_;
      for (auto& kv : cb) {
        std::vector<uint32_t> v(n);
        uint32_t t = 1;
        for (size_t k = 0; k < n; k++) { v[k] = mul(kv.second[k], t); t = mul(t, s); }
        fft_dif(v.data(), n); bit_reverse(v.data(), n);
        vb_[kv.first] = v;
      }
      for (auto& kv : ce) {
        std::vector<E6> v(n);
        uint32_t t = 1;
        for (size_t k = 0; k < n; k++) { v[k] = e6_mul_base(kv.second[k], t); t = mul(t, s); }
        fft_dif_e6(v.data(), n); bit_reverse_e6(v.data(), n);
        ve_[kv.first] = v;
      }
      uint32_t zinv = inv(sub(pow(s, n), 1));
      auto colval = [&](uint32_t c, size_t r) -> Val {
        if (pg.columns[c].field == 0) return vb(vb_.at(c)[r]);
        return ve(ve_.at(c)[r]);
      };
#pragma omp parallel for schedule(static)
      for (size_t j = 0; j < n; j++) {
        std::vector<Val> sc(nodes.size());
        E6 v = as_e6(eval(order, (uint32_t)fold_root[m], j, n, colval, sc));
        num[rho * j + i] = e6_mul_base(v, zinv);
      }
    }
    ifft_dif_e6(num.data(), big);
    bit_reverse_e6(num.data(), big);
    uint32_t gi = inv(g), acc = 1;
    for (size_t k = 0; k < big; k++) { num[k] = e6_mul_base(num[k], acc); acc = mul(acc, gi); }
    std::vector<std::vector<E6>> chunks(rho);
    for (uint32_t c = 0; c < rho; c++) {
      std::vector<E6> ch(num.begin() + c * n, num.begin() + (c + 1) * n);
      fft_dif_e6(ch.data(), n);
      bit_reverse_e6(ch.data(), n);
      chunks[c] = std::move(ch);
    }
    return chunks;
  }
  // Quotients of every module with a relation: modules run in parallel
  // (largest first), each serially inside.
  void quotients() {
    std::vector<uint32_t> ms;
    for (uint32_t m : mod_order) if (chunk_count(m)) ms.push_back(m);
    std::stable_sort(ms.begin(), ms.end(), [&](uint32_t a, uint32_t b) { return mod_n(a) > mod_n(b); });
    std::vector<std::vector<std::vector<E6>>> res(ms.size());
#pragma omp parallel for schedule(dynamic) if (ms.size() > 1)
    for (size_t i = 0; i < ms.size(); i++) res[i] = quotient(ms[i]);
    for (size_t i = 0; i < ms.size(); i++) {
      const uint32_t m = ms[i];
      const size_t n = mod_n(m);
      for (uint32_t c = 0; c < res[i].size(); c++) {
        if (root_ext[m]) air_ext[{m, c}] = res[i][c];
        else {
          std::vector<uint32_t> b(n);
          for (size_t k = 0; k < n; k++) b[k] = res[i][c][k].c[0];
          air_base[{m, c}] = b;
        }
      }
    }
  }

  // ---------------------------------------------------------- open helpers
  // L_i(zeta) = (zeta^n - 1)/n * w^i / (zeta - w^i)  (internal/poly/utils.go:66-104)
  std::vector<E6> lagranges_at(const E6& z, size_t n) {
    std::vector<E6> res(n);
    const uint32_t w = root_of_unity(n);
    const E6 common = e6_mul_base(e6_sub(e6_pow(z, n), e6_one()), inv((uint32_t)(n % P)));
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; i++) {
      const uint32_t wi = pow(w, i);
      res[i] = e6_mul(e6_mul_base(common, wi), e6_inv(e6_sub(z, e6_from_base(wi))));
    }
    return res;
  }
  // sum_i L_{(i - s) mod n}(zeta) P[i]  (internal/poly/ext.go:84-104)
  static E6 eval_lagrange(const uint32_t* p, const std::vector<E6>& L, size_t s) {
    size_t n = L.size();
    E6 acc = e6_zero();
    for (size_t i = 0; i < n; i++) acc = e6_add(acc, e6_mul_base(L[(n + i - s) % n], p[i]));
    return acc;
  }
  static E6 eval_lagrange_e6(const E6* p, const std::vector<E6>& L, size_t s) {
    size_t n = L.size();
    E6 acc = e6_zero();
    for (size_t i = 0; i < n; i++) acc = e6_add(acc, e6_mul(L[(n + i - s) % n], p[i]));
    return acc;
  }
  std::vector<int> shifts_of(const TreeL& t, uint32_t c) {
    if (t.air) return {0};
    auto it = col_shifts.find(c);
    return it == col_shifts.end() ? std::vector<int>{} : it->second;
  }

  struct GroupCV { std::vector<std::vector<E6>> b, e; };
  // fold: (p+q)/2 + alpha (p-q)/(2x), x^-1 = w_n^-bitrev(i, n/2) (internal/fri/fri.go:1177-1198)
  static std::vector<E6> fold(const std::vector<E6>& layer, const E6& alpha) {
    size_t n = layer.size(), half = n / 2;
    int lg = 0; while ((1ull << lg) < half) lg++;
    uint32_t winv = inv(root_of_unity(n)), inv2 = inv(2);
    std::vector<E6> next(half);
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < half; i++) {
      uint32_t xi = pow(winv, bitrev((uint32_t)i, lg));
      E6 p = layer[2 * i], q = layer[2 * i + 1];
      E6 s = e6_mul_base(e6_add(p, q), inv2);
      E6 d = e6_mul(e6_mul_base(e6_mul_base(e6_sub(p, q), inv2), xi), alpha);
      next[i] = e6_add(s, d);
    }
    return next;
  }
  static std::vector<Digest> ext_leaves(const std::vector<E6>& layer) {
    Source s; s.rows = layer.size(); s.e.push_back(layer);
    return hash_leaf_pairs(s);
  }

  // ---------------------------------------------------------- prove
  std::vector<uint8_t> prove(const uint32_t* const* witness) {
    setup(witness);
    Writer W;
    uint32_t R = pg.n_rounds;
    for (uint32_t r = 0; r < R; r++) fs.new_challenge(coin_name(r));
    fs.new_challenge("__zeta");
    std::string first = R > 0 ? coin_name(0) : "__zeta";
    fs.bind(first, string_to_elements(0x48415348, "poseidon2"));
    {
      std::vector<uint32_t> sz = {0x53495a45, (uint32_t)mod_order.size()};
      for (uint32_t m : mod_order) sz.push_back((uint32_t)mod_n(m));
      fs.bind(first, sz);
    }
    // setup tree: precommitted, its root bound to the first challenge and
    // kept out of the proof's commitments (prover/prover.go:175-229)
    size_t tree_idx = 0;
    if (!trees.empty() && trees[0].setup) {
      committed.push_back(commit(tree_groups(trees[0])));
      setup_root = committed.back().tree.root();
      fs.bind(first, setup_root.v, 8);
      tree_idx = 1;
    }
    // rounds: steps, commit, bind root, sample (prover/prover.go:360-411)
    coins.assign(R, e6_zero());
    for (uint32_t r = 0; r < R; r++) {
      for (const PStep& st : pg.steps) if (st.round == r) run_step(st);
      if (tree_idx < trees.size() && !trees[tree_idx].air && trees[tree_idx].round == (int)r) {
        committed.push_back(commit(tree_groups(trees[tree_idx])));
        Digest root = committed.back().tree.root();
        commitments.push_back(root);
        fs.bind(coin_name(r), root.v, 8);
        tree_idx++;
      }
      // BindExposedValues (prover/prover.go:386-396): in step order, entry
      // index then the value as six elements (board/logup.go:218-225)
      for (const PStep& st : pg.steps) {
        if (st.round != r || (st.type != STEP_LOGUP && st.type != STEP_RATIO)) continue;
        uint32_t w[7] = {0};
        for (int k = 0; k < 6; k++) w[1 + k] = exposed[st.exposed].c[k];
        fs.bind(coin_name(r), w, 7);
      }
      coins[r] = digest_to_e6(fs.compute(coin_name(r)));
    }
    // AIR quotients (prover/prover.go:461-561)
    quotients();
    if (tree_idx < trees.size() && trees[tree_idx].air) {
      committed.push_back(commit(tree_groups(trees[tree_idx])));
      Digest root = committed.back().tree.root();
      commitments.push_back(root);
      fs.bind("__zeta", root.v, 8);
    }
    zeta = digest_to_e6(fs.compute("__zeta"));

    // claimed values (internal/fri/values.go:46-110)
    std::map<size_t, std::vector<E6>> lag;
    std::vector<std::vector<GroupCV>> cv(trees.size());
    std::vector<std::pair<size_t, size_t>> tg;  // (tree, group), evaluated in parallel
    for (size_t t = 0; t < trees.size(); t++) {
      cv[t].resize(trees[t].groups.size());
      for (size_t g = 0; g < trees[t].groups.size(); g++) {
        const size_t n = mod_n(trees[t].groups[g].module);
        if (!lag.count(n)) lag[n] = lagranges_at(zeta, n);
        tg.push_back({t, g});
      }
    }
#pragma omp parallel for schedule(dynamic)
    for (size_t q = 0; q < tg.size(); q++) {
      const size_t t = tg[q].first;
      {
        const Group& g = trees[t].groups[tg[q].second];
        const auto& L = lag.at(mod_n(g.module));
        GroupCV gv;
        for (uint32_t c : g.bcols) {
          const uint32_t* p = trees[t].air ? air_base.at({g.module, c}).data() : base.at(c).data();
          std::vector<E6> vals;
          for (int s : shifts_of(trees[t], c)) vals.push_back(eval_lagrange(p, L, (size_t)s));
          gv.b.push_back(vals);
        }
        for (uint32_t c : g.ecols) {
          const E6* p = trees[t].air ? air_ext.at({g.module, c}).data() : ext.at(c).data();
          std::vector<E6> vals;
          for (int s : shifts_of(trees[t], c)) vals.push_back(eval_lagrange_e6(p, L, (size_t)s));
          gv.e.push_back(vals);
        }
        cv[t][tg[q].second] = gv;
      }
    }
    // DEEP classes = modules in sorted order (internal/protocol/layout.go:90-103,
    // internal/fri/deep_classes.go:64-124)
    std::vector<uint32_t> classes;
    for (uint32_t m : mod_order) {
      bool has = false;
      for (auto& t : trees) for (auto& g : t.groups) if (g.module == m) has = true;
      if (has) classes.push_back(m);
    }
    fs.new_challenge("alpha_DEEP");
    for (uint32_t m : classes)
      for (size_t t = 0; t < trees.size(); t++)
        for (size_t g = 0; g < trees[t].groups.size(); g++) {
          if (trees[t].groups[g].module != m) continue;
          for (auto& vals : cv[t][g].b) for (auto& v : vals) fs.bind("alpha_DEEP", v.c, 6);
          for (auto& vals : cv[t][g].e) for (auto& v : vals) fs.bind("alpha_DEEP", v.c, 6);
        }
    E6 alpha = digest_to_e6(fs.compute("alpha_DEEP"));

    // DEEP codewords (internal/fri/deep.go:71-266)
    std::vector<std::vector<E6>> deep(classes.size());
    // classes are independent: they run in parallel, each serially inside
    // (with few classes, serially with the rows in parallel)
#pragma omp parallel for schedule(dynamic) if (classes.size() >= 4)
    for (size_t ci = 0; ci < classes.size(); ci++) {
      uint32_t m = classes[ci];
      size_t n = mod_n(m);
      uint32_t w = root_of_unity(n);
      struct Term { size_t point; E6 scaled; };
      struct Bundle { const uint32_t* b; const E6* e; E6 scale; std::vector<Term> terms; };
      std::vector<Bundle> bundles;
      std::vector<E6> points;
      E6 run = e6_one();
      auto add_terms = [&](Bundle& bu, const std::vector<int>& shifts, const std::vector<E6>& vals) {
        for (size_t k = 0; k < shifts.size(); k++) {
          E6 z = e6_mul_base(zeta, pow(w, (uint64_t)shifts[k]));
          size_t pi = points.size();
          for (size_t q = 0; q < points.size(); q++) if (e6_eq(points[q], z)) { pi = q; break; }
          if (pi == points.size()) points.push_back(z);
          bu.terms.push_back({pi, e6_mul(bu.scale, vals[k])});
        }
      };
      for (size_t t = 0; t < trees.size(); t++)
        for (size_t g = 0; g < trees[t].groups.size(); g++) {
          const Group& G = trees[t].groups[g];
          if (G.module != m) continue;
          for (size_t i = 0; i < G.bcols.size(); i++) {
            Bundle bu; bu.b = trees[t].air ? air_base.at({m, G.bcols[i]}).data() : base.at(G.bcols[i]).data(); bu.e = nullptr; bu.scale = run;
            add_terms(bu, shifts_of(trees[t], G.bcols[i]), cv[t][g].b[i]);
            bundles.push_back(bu);
            run = e6_mul(run, alpha);
          }
          for (size_t i = 0; i < G.ecols.size(); i++) {
            Bundle bu; bu.b = nullptr; bu.e = trees[t].air ? air_ext.at({m, G.ecols[i]}).data() : ext.at(G.ecols[i]).data(); bu.scale = run;
            add_terms(bu, shifts_of(trees[t], G.ecols[i]), cv[t][g].e[i]);
            bundles.push_back(bu);
            run = e6_mul(run, alpha);
          }
        }
      std::vector<E6> dq(n, e6_zero());
#pragma omp parallel for schedule(static)
      for (size_t x = 0; x < n; x++) {
        uint32_t wx = pow(w, x);
        std::vector<E6> numer(points.size(), e6_zero());
        for (auto& bu : bundles) {
          E6 sp = bu.b ? e6_mul_base(bu.scale, bu.b[x]) : e6_mul(bu.scale, bu.e[x]);
          for (auto& tm : bu.terms) numer[tm.point] = e6_sub(e6_add(numer[tm.point], tm.scaled), sp);
        }
        E6 acc = e6_zero();
        for (size_t q = 0; q < points.size(); q++)
          acc = e6_add(acc, e6_mul(numer[q], e6_inv(e6_sub(points[q], e6_from_base(wx)))));
        dq[x] = acc;
      }
      deep[ci] = rs_encode_e6(dq.data(), n, RATE * n);
    }

    // FRI (internal/fri/fri.go:352-365,606-736)
    std::vector<size_t> class_at(classes.size());
    for (size_t i = 0; i < class_at.size(); i++) class_at[i] = i;
    std::stable_sort(class_at.begin(), class_at.end(), [&](size_t a, size_t b) { return mod_n(classes[a]) > mod_n(classes[b]); });
    size_t L = class_at.size();
    std::vector<size_t> lvl_d(L);
    std::vector<const std::vector<E6>*> lvl(L);
    for (size_t l = 0; l < L; l++) { lvl_d[l] = mod_n(classes[class_at[l]]); lvl[l] = &deep[class_at[l]]; }
    const int NR = MAX_LOG;
    auto lg2 = [](uint64_t x) { int k = 0; while ((1ull << k) < x) k++; return k; };
    int r0 = lg2(((uint64_t)1 << MAX_LOG) / lvl_d[0]);
    if (r0 >= NR) throw std::runtime_error("FRI: first level too small");
    for (size_t l = 1; l < L; l++) fs.new_challenge("fri_level_" + std::to_string(l) + "_gamma");
    for (int j = 0; j < NR; j++) fs.new_challenge("fri_fold_" + std::to_string(j));
    for (uint32_t k = 0; k < num_queries; k++) fs.new_challenge("fri_query_" + std::to_string(k));
    std::vector<std::vector<Digest>> lleaves(L);
    for (size_t l = 0; l < L; l++) lleaves[l] = ext_leaves(*lvl[l]);
    std::vector<Injection> linj;
    for (size_t l = 1; l < L; l++) linj.push_back(Injection{lleaves[l]});
    Tree levels_tree = build_tree(lleaves[0], linj);
    std::vector<E6> gam(L);
    for (size_t l = 1; l < L; l++) {
      std::string nm = "fri_level_" + std::to_string(l) + "_gamma";
      if (l == 1) fs.bind(nm, levels_tree.root().v, 8);
      gam[l] = digest_to_e6(fs.compute(nm));
    }
    Digest zero; memset(zero.v, 0, sizeof zero.v);
    for (int j = 0; j < r0; j++) {
      fs.bind("fri_fold_" + std::to_string(j), zero.v, 8);
      fs.compute("fri_fold_" + std::to_string(j));
    }
    std::vector<std::vector<E6>> layers(NR + 1);
    std::vector<Tree> ftrees(NR);
    std::vector<Digest> fri_roots;
    std::vector<E6> running = *lvl[0];
    for (int j = r0; j < NR; j++) {
      if (j == r0) layers[j] = *lvl[0];
      for (size_t l = 1; l < L; l++) {
        if (lg2(((uint64_t)1 << MAX_LOG) / lvl_d[l]) != j) continue;
#pragma omp parallel for schedule(static)
        for (size_t k = 0; k < running.size(); k++) running[k] = e6_add(running[k], e6_mul((*lvl[l])[k], gam[l]));
      }
      if (j > r0) layers[j] = running;
      ftrees[j] = j == r0 ? levels_tree : build_tree(ext_leaves(running), {});
      Digest root = ftrees[j].root();
      std::string nm = "fri_fold_" + std::to_string(j);
      fs.bind(nm, root.v, 8);
      E6 a = digest_to_e6(fs.compute(nm));
      if (j > r0) fri_roots.push_back(root);
      running = fold(running, a);
    }
    {
      std::vector<uint32_t> fin = {0x45585450, (uint32_t)running.size()};
      for (auto& v : running) for (int i = 0; i < 6; i++) fin.push_back(v.c[i]);
      fs.bind("fri_query_0", fin);
    }
    struct QL { uint32_t row; E6 p, q; MerklePath path; bool has_path; };
    std::vector<std::vector<QL>> fq(num_queries), lq(L > 1 ? L - 1 : 0, std::vector<QL>(num_queries));
    std::vector<uint64_t> positions(num_queries);
    for (uint32_t k = 0; k < num_queries; k++) {
      Digest c = fs.compute("fri_query_" + std::to_string(k));
      uint64_t s = (((uint64_t)c.v[0] << 31) ^ (uint64_t)c.v[1]) % N_FRI;
      positions[k] = s;
      if (k + 1 < num_queries) fs.bind("fri_query_" + std::to_string(k + 1), c.v, 8);
      for (int j = r0; j < NR; j++) {
        uint32_t row = (uint32_t)(s >> j), lo = row & ~1u;
        QL q; q.row = row; q.p = layers[j][lo]; q.q = layers[j][lo + 1];
        q.path = open_path(ftrees[j], lo / 2); q.has_path = true;
        if (j == r0) q.path.injection_leaves.clear();
        fq[k].push_back(q);
      }
      for (size_t l = 1; l < L; l++) {
        int jl = lg2(((uint64_t)1 << MAX_LOG) / lvl_d[l]);
        uint32_t row = (uint32_t)(s >> jl), lo = row & ~1u;
        QL q; q.row = row; q.p = (*lvl[l])[lo]; q.q = (*lvl[l])[lo + 1]; q.has_path = false;
        q.path.leaf_idx = 0;
        lq[l - 1][k] = q;
      }
    }

    // ---- serialize (canonical encoding; see loom_gpu.h)
    W.str("poseidon2");
    {  // exposed values, by name: name, entries (index, field kind 1 = ext, six words)
      std::vector<size_t> ord(exposed.size());
      for (size_t i = 0; i < ord.size(); i++) ord[i] = i;
      std::sort(ord.begin(), ord.end(), [&](size_t a, size_t b) { return exposed_names[a] < exposed_names[b]; });
      W.u32((uint32_t)ord.size());
      for (size_t i : ord) {
        W.str(exposed_names[i]);
        W.u32(1);
        W.u32(0);
        W.u32(1);
        for (int k = 0; k < 6; k++) W.u32(exposed[i].c[k]);
      }
    }
    W.u32((uint32_t)commitments.size());
    for (auto& d : commitments) W.dg(d);
    W.u32((uint32_t)trees.size());
    for (size_t t = 0; t < trees.size(); t++) {
      W.u32((uint32_t)cv[t].size());
      for (auto& gv : cv[t]) {
        W.u32((uint32_t)gv.b.size());
        for (auto& vals : gv.b) { W.u32((uint32_t)vals.size()); for (auto& v : vals) W.e6(v); }
        W.u32((uint32_t)gv.e.size());
        for (auto& vals : gv.e) { W.u32((uint32_t)vals.size()); for (auto& v : vals) W.e6(v); }
      }
    }
    auto wpath = [&](const MerklePath& p) {
      W.u32(p.leaf_idx);
      W.u32((uint32_t)p.siblings.size()); for (auto& d : p.siblings) W.dg(d);
      W.u32((uint32_t)p.injection_leaves.size()); for (auto& d : p.injection_leaves) W.dg(d);
    };
    auto wql = [&](const QL& q) {
      W.u32(1); W.u32(q.row); W.e6(q.p); W.e6(q.q);
      if (q.has_path) wpath(q.path); else { W.u32(0); W.u32(0); W.u32(0); }
    };
    W.dg(levels_tree.root());
    W.u32((uint32_t)lq.size());
    for (auto& set : lq) { W.u32((uint32_t)set.size()); for (auto& q : set) wql(q); }
    W.u32((uint32_t)fri_roots.size());
    for (auto& d : fri_roots) W.dg(d);
    W.u32(1);  // final field: ext
    W.u32((uint32_t)running.size());
    for (auto& v : running) W.e6(v);
    W.u32(num_queries);
    for (auto& q : fq) { W.u32((uint32_t)q.size()); for (auto& x : q) wql(x); }
    W.u32(0);  // proofs of work
    W.u32(num_queries);
    for (uint32_t k = 0; k < num_queries; k++) {
      W.u32((uint32_t)committed.size());
      for (auto& c : committed) {
        uint64_t s = positions[k];
        auto wrow = [&](const Source& src, size_t row) {
          W.u32((uint32_t)src.b.size()); for (auto& col : src.b) W.el(col[row]);
          W.u32((uint32_t)src.e.size()); for (auto& col : src.e) W.e6(col[row]);
        };
        const Source& top = c.sources[0];
        size_t trow = (size_t)(s >> (lg2(N_FRI) - lg2(top.rows))), tlo = trow & ~(size_t)1;
        wrow(top, tlo); wrow(top, tlo + 1);
        wpath(open_path(c.tree, tlo / 2));
        W.u32((uint32_t)(c.sources.size() - 1));
        for (size_t k2 = 1; k2 < c.sources.size(); k2++) {
          const Source& src = c.sources[k2];
          size_t row = (size_t)(s >> (lg2(N_FRI) - lg2(src.rows))), lo = row & ~(size_t)1;
          wrow(src, lo); wrow(src, lo + 1);
        }
      }
    }
    return W.b;
  }
};

}  // namespace

}  // namespace orc
