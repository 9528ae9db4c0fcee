// The prove flow on one device (prover/prover.go:142-719): rounds with
// grand-product steps and commits, AIR quotients, claimed values, DEEP
// codewords, multi-degree FRI and query openings.  The transcript runs on the
// host; roots and openings are read back from the device.
#pragma once
#include <set>

#include "commit.cuh"
#include "xjit.cuh"

namespace lg {

constexpr int MAX_LOG_MODULE = 22;  // internal/constants/const.go:27-32
constexpr int LOG_N_FRI = MAX_LOG_MODULE + RATE_LOG;
const int NEG_INF = -1000000;

inline std::string coin_name(uint32_t r) { return "challenge@loom_" + std::to_string(r); }

struct ProveStats { double ms_total = 0; };



// The bytecode of one compile site (a step's expressions, a module's folded
// relation) depends only on the program and on the order in which the site's
// columns first reach its lane table.  A later prove of the same program
// feeds the recorded columns to a fresh table in that order, which rebuilds
// the same lane indices, and reuses the code and its device copy.
struct CodeSet {
  std::vector<XCode> xc;
  std::vector<XProgram> dev;   // device copies, in xc order
  std::vector<uint32_t> cols;  // columns in first-use order
  DBufP code;                  // every xc back to back (kept across proves)
  // The kernel compiled from xc at run time (xjit.cuh: the quotient's program,
  // or a grand product's numerator and denominator), looked up once: later
  // proves skip generating its source to find it in the compile cache.
  mutable bool jit_done = false;
  mutable CUfunction jit = nullptr;
};
// A program's precommitted setup tree (lg_setup; setup/setup.go:68-124): the
// committed LDE and tree, the setup columns' values and coefficients, and the
// root the verifier holds as its key.  Kept on the context with the program.
struct SetupData {
  Committed committed;
  Digest root;
  std::map<uint32_t, DBufP> values;            // setup column -> Lagrange values
  std::map<uint32_t, const uint32_t*> coef;    // setup column -> coefficient lane 0 (in committed)
};
struct ProgCache {
  std::vector<uint32_t> words;  // the program descriptor, compared in full
  std::map<std::string, std::shared_ptr<CodeSet>> sites;
  std::shared_ptr<SetupData> setup;
};

struct Prover {
  Ctx& c;
  Program pg;
  uint32_t num_queries;
  Transcript fs;
  std::vector<E6> coins;
  // Exposed values (logup totals, in step order): Montgomery E6 once read back.
  std::vector<E6> exposed;
  std::vector<char> exposed_ready;
  DBufP exposed_d;  // 6 words per exposed value, written by k_logup_finish
  DBufP coins_dev;
  std::vector<uint32_t> mod_order;
  std::vector<int> fold_root, degree;
  std::vector<bool> root_ext;
  std::map<uint32_t, std::vector<int>> col_shifts;

  // column data on the device: lane pointer = buf + w * n
  std::map<uint32_t, DBufP> col_buf;
  DBufP witness_dev;  // host witness columns, uploaded into one buffer
  bool upload_pending = false;  // late columns of a split upload still on the side stream (await_upload)
  std::map<uint32_t, const uint32_t*> col_coef;  // committed columns: coefficient lane 0

  struct Group { uint32_t module; std::vector<uint32_t> bcols, ecols; };
  struct TreeL { bool air; int round; std::vector<Group> groups; bool setup = false; };
  std::vector<TreeL> trees;
  std::vector<Committed> committed;
  std::vector<Digest> commitments;
  std::map<uint32_t, DBufP> chunk_coef;  // module -> chunks (d * lanes + w) * n
  E6 zeta;
  // Device copies of the challenges the kernels read: slot r (8 words) for
  // round coin r, slot n_rounds for __zeta.  With dev_fs (the whole prove,
  // lg_prove) the device computes them itself from roots and exposed values
  // still in device memory (k_fs_chain), and the host transcript replays and
  // checks them at the next read-back (sync_transcript); otherwise
  // set_challenge uploads the caller's values.
  // Slot n_rounds + 1 holds zeros (the entry-index word of exposed bindings).
  DBufP fs_slots;
  bool dev_fs = false;
  struct PendingRoot { size_t commitment, tree; };      // root still on the device
  struct PendingCoin { uint32_t round; int commitment; };  // round n_rounds: __zeta
  std::vector<PendingRoot> pending_roots;
  std::vector<PendingCoin> pending_coins;
  uint32_t* fs_slot(uint32_t k) const { return fs_slots->p + 8 * (size_t)k; }
  // challenges queued for the device (k_fs_chain)
  struct FsQueue {
    struct Seg { const uint32_t* dev; size_t off; uint32_t len, moff; };  // dev null: consts[off, off + len)
    std::vector<uint32_t> consts;
    std::vector<Seg> segs;
    std::vector<FsChal> chs;
    uint32_t words = 0;  // message words of the queued challenges
  };
  using DevWords = std::vector<std::pair<const uint32_t*, uint32_t>>;
  std::vector<char> fold_dev;               // fold challenges up to r0 the device computed (lg_prove)

  ProgCache* prog = nullptr;  // compiled code of this program, kept on the context
  std::shared_ptr<ProgCache> prog_keep;  // ... and alive while this prove lasts

  // ---- state of the phases (prove_flow.cuh), in the order they run
  struct Poly { size_t t, g; bool ext; const uint32_t* coef; uint32_t logn; std::vector<int> shifts; };
  size_t tree_next = 0;                     // next entry of `trees` to commit
  std::vector<char> coin_ready;             // per round: its challenge is known
  bool zeta_ready = false, alpha_ready = false;
  E6 alpha;
  std::vector<std::vector<std::vector<Poly>>> polys;                  // [tree][group] base then ext polys
  std::vector<std::vector<std::vector<std::vector<E6>>>> cv;          // claimed values [tree][group][poly][shift]
  std::vector<uint32_t> classes;            // DEEP classes: modules with committed groups, layout order
  std::vector<DBufP> deep;                  // DEEP codeword per class (6 lanes x 4n)
  std::vector<DBufP> deep_den;              // per class: 1/(z_s - x) per point (k_deep_den), or empty
  bool den_pending = false;                 // k_deep_den queued on the side stream, not yet joined
  // FRI (internal/fri/fri.go:352-365,606-736)
  size_t L = 0;                             // levels, sorted by size (descending, stable)
  int NR = 0, r0 = 0;                       // rounds; the first round with a layer
  std::vector<uint32_t> lvl_log;
  std::vector<DBufP> lvl;
  TreeDev levels_tree;
  std::vector<E6> gam;                      // level weights (gam[0] unused)
  DBufP gam_d;                              // their device slots (8 words each)
  std::vector<char> gam_ready;
  std::vector<DBufP> layers;                // layer j (E6 lanes), r0 <= j < NR
  std::vector<TreeDev> ftrees;
  std::vector<Digest> fri_roots;            // layer roots after the first
  DBufP chal;                               // fold challenge j at chal + 8 j (digest words)
  std::vector<char> chal_ready;
  DBufP running;                            // the layer being folded
  size_t nj = 0;                            // its length
  int fri_next = -1;                        // next round to fold (-1: levels not committed)
  std::vector<uint32_t> final_poly;         // 6 lanes of nj words, once read back
  struct OpenPrep;                          // the openings' word map (prove_flow.cuh)
  std::shared_ptr<OpenPrep> oplan;  // (shared_ptr: complete only in prove_flow.cuh)

  // A prover dropped with the DEEP denominators still queued (a session
  // released before its DEEP phase) orders the frees of its buffers, which
  // run on the main stream, after that work.
  ~Prover() {
    if (den_pending) cudaStreamWaitEvent(c.stream, c.join_ev, 0);
    if (upload_pending) cudaStreamWaitEvent(c.stream, c.upload_ev, 0);
  }
  Prover(const Prover&) = delete;
  Prover& operator=(const Prover&) = delete;
  Prover(Ctx& ctx, const uint32_t* words, size_t nwords, uint32_t q) : c(ctx), num_queries(q) {
    pg = parse_program(words, nwords);
    if (q == 0) throw Error(LG_ERR_INVALID, "num_queries must be positive");
    if (q > 65535) throw Error(LG_ERR_UNSUPPORTED, "num_queries above 65535 is not supported by this build");
    auto& L = c.programs;
    auto it = std::find_if(L.begin(), L.end(), [&](const std::shared_ptr<ProgCache>& e) {
      return e->words.size() == nwords && std::equal(e->words.begin(), e->words.end(), words);
    });
    if (it != L.end()) {
      L.splice(L.begin(), L, it);
    } else {
      auto e = std::make_shared<ProgCache>();
      e->words.assign(words, words + nwords);
      L.push_front(e);
      while (L.size() > Ctx::MAX_PROGRAMS) L.pop_back();
    }
    prog_keep = L.front();
    prog = prog_keep.get();
  }

  // The bytecode of `roots` compiled in order against one lane table
  // (lane_of), from the program's cache when this site was compiled before.
  // The run-time compiled kernel of a cached code set (null: the interpreter
  // runs it), found once per code set.
  static CUfunction jit_of(const CodeSet& cs, bool grand_product) {
    if (!cs.jit_done) {
      cs.jit = grand_product ? xjit_gp(cs.xc.at(0), cs.xc.at(1)) : xjit_quotient(cs.xc.at(0));
      cs.jit_done = true;
    }
    return cs.jit;
  }
  template <class LaneOf> const CodeSet& compiled(const std::string& site, LaneOf& lane_of, const std::vector<uint32_t>& roots) {
    auto it = prog->sites.find(site);
    if (it != prog->sites.end()) {
      for (uint32_t col : it->second->cols) lane_of(col);
      return *it->second;
    }
    auto cs = std::make_shared<CodeSet>();
    std::vector<char> seen(pg.columns.size(), 0);
    auto rec = [&](uint32_t col) -> uint32_t {
      if (!seen[col]) { seen[col] = 1; cs->cols.push_back(col); }
      return lane_of(col);
    };
    for (uint32_t r : roots) cs->xc.push_back(compile_expr(r, rec));
    std::vector<XInst> all;
    std::vector<size_t> off;
    for (auto& x : cs->xc) { off.push_back(all.size()); all.insert(all.end(), x.code.begin(), x.code.end()); }
    {
      ArenaScope kept(nullptr);  // outlives this prove
      cs->code = upload_vec(c, all);
    }
    for (size_t i = 0; i < cs->xc.size(); i++) {
      const XCode& x = cs->xc[i];
      cs->dev.push_back(XProgram{(const XInst*)cs->code->p + off[i], (uint32_t)x.code.size(), x.n_regs, x.result, x.result_ext});
    }
    prog->sites[site] = cs;
    return *cs;
  }
  size_t step_index(const Step* st) const { return (size_t)(st - pg.steps.data()); }

  size_t mod_n(uint32_t m) const { return (size_t)1 << pg.modules[m].log_n; }
  uint32_t lanes_of(uint32_t col) const { return pg.columns[col].field ? 6 : 1; }
  const uint32_t* lane_ptr(uint32_t col, uint32_t w) const {
    return col_buf.at(col)->p + (size_t)w * mod_n(pg.columns[col].module);
  }

  // ------------------------------------------------------------ DAG helpers
  uint32_t push(uint32_t op, uint32_t a, uint32_t b) { pg.nodes.push_back({op, a, b}); return (uint32_t)pg.nodes.size() - 1; }
  int node_degree(uint32_t id, std::vector<int>& memo) {
    if (memo[id] != INT32_MIN) return memo[id];
    const Node& x = pg.nodes[id];
    int d = 0;
    switch (x.op) {
      case OP_COL: d = 1; break;
      case OP_EXPAVG: d = 1; break;  // a verifier column (internal/dag/dag.go:1536)
      case OP_EXPVAL: d = 0; break;  // a constant (times L_0 it is the sparse column)
      case OP_COIN: d = 0; break;
      case OP_CONST: d = x.a % P == 0 ? NEG_INF : 0; break;
      case OP_ADD: case OP_SUB: d = std::max(node_degree(x.a, memo), node_degree(x.b, memo)); break;
      default: {
        int l = node_degree(x.a, memo), r = node_degree(x.b, memo);
        d = (l == NEG_INF || r == NEG_INF) ? NEG_INF : l + r;
      }
    }
    return memo[id] = d;
  }
  bool node_ext(uint32_t id) const {
    const Node& x = pg.nodes[id];
    if (x.op == OP_COL) return pg.columns[x.a].field == 1;
    if (x.op == OP_COIN || x.op == OP_EXPAVG || x.op == OP_EXPVAL) return true;
    if (x.op == OP_CONST) return false;
    return false;  // combined by the caller through ext_of
  }
  std::vector<char> ext_of;  // per node
  void compute_ext() {
    ext_of.assign(pg.nodes.size(), 0);
    for (size_t i = 0; i < pg.nodes.size(); i++) {
      const Node& x = pg.nodes[i];
      if (is_binary(x.op)) ext_of[i] = ext_of[x.a] || ext_of[x.b];
      else ext_of[i] = node_ext((uint32_t)i);
    }
  }
  // Marks the nodes under id in `seen`; appends each newly marked one to
  // `order` when given.
  void collect(uint32_t id, std::vector<char>& seen, std::vector<uint32_t>* order = nullptr) {
    std::vector<uint32_t> st = {id};
    while (!st.empty()) {
      uint32_t x = st.back();
      st.pop_back();
      if (seen[x]) continue;
      seen[x] = 1;
      if (order) order->push_back(x);
      if (is_binary(pg.nodes[x].op)) { st.push_back(pg.nodes[x].a); st.push_back(pg.nodes[x].b); }
    }
  }

  // Compiles the sub-DAG under `root` into register bytecode.  lane_of(col)
  // gives the first lane index the kernel reads for that column.
  template <class LaneOf> XCode compile_expr(uint32_t root, LaneOf lane_of) {
    std::vector<char> seen(pg.nodes.size(), 0);
    collect(root, seen);
    // Evaluation order: post-order from the root, the child that needs more
    // registers first (Sethi-Ullman), so a long sum of relations folded by
    // Horner keeps one accumulator live instead of every relation's value.
    std::vector<int> need(pg.nodes.size(), 0);
    for (uint32_t i = 0; i < pg.nodes.size(); i++) {
      if (!seen[i]) continue;
      const Node& x = pg.nodes[i];
      if (!is_binary(x.op)) { need[i] = 1; continue; }
      int na = need[x.a], nb = need[x.b];
      need[i] = na == nb ? na + 1 : std::max(na, nb);
    }
    std::vector<uint32_t> order;
    {
      std::vector<char> done(pg.nodes.size(), 0);
      std::vector<std::pair<uint32_t, int>> st = {{root, 0}};
      while (!st.empty()) {
        auto [x, state] = st.back();
        st.pop_back();
        if (done[x]) continue;
        const Node& nd = pg.nodes[x];
        if (state == 1 || !is_binary(nd.op)) {
          done[x] = 1;
          order.push_back(x);
          continue;
        }
        st.push_back({x, 1});
        uint32_t first = need[nd.a] >= need[nd.b] ? nd.a : nd.b, second = first == nd.a ? nd.b : nd.a;
        st.push_back({second, 0});
        st.push_back({first, 0});
      }
    }
    std::vector<int> last(pg.nodes.size(), -1);
    for (size_t k = 0; k < order.size(); k++) {
      const Node& x = pg.nodes[order[k]];
      if (is_binary(x.op)) { last[x.a] = (int)k; last[x.b] = (int)k; }
    }
    last[root] = (int)order.size();
    std::vector<int> reg(pg.nodes.size(), -1);
    std::vector<uint32_t> free_regs;
    XCode xc;
    for (size_t k = 0; k < order.size(); k++) {
      uint32_t id = order[k];
      const Node& x = pg.nodes[id];
      XInst in{};
      // free operand registers whose last use is here (after reading them)
      std::vector<uint32_t> to_free;
      if (is_binary(x.op)) {
        if (last[x.a] == (int)k) to_free.push_back((uint32_t)reg[x.a]);
        if (last[x.b] == (int)k && x.b != x.a) to_free.push_back((uint32_t)reg[x.b]);
      }
      uint32_t d;
      if (!free_regs.empty()) { d = free_regs.back(); free_regs.pop_back(); }
      else d = xc.n_regs++;
      in.d = (uint8_t)d;
      bool ea = is_binary(x.op) && ext_of[x.a], eb = is_binary(x.op) && ext_of[x.b];
      uint32_t ra = is_binary(x.op) ? (uint32_t)reg[x.a] : 0, rb = is_binary(x.op) ? (uint32_t)reg[x.b] : 0;
      switch (x.op) {
        case OP_COL:
          in.op = pg.columns[x.a].field ? X_LOAD_E : X_LOAD_B;
          in.imm = lane_of(x.a);
          in.shift = (int32_t)x.b;
          break;
        case OP_COIN: in.op = X_COIN; in.imm = x.a; break;
        // the kernels' coin table: round coins, exposed averages, exposed values
        case OP_EXPAVG: in.op = X_COIN; in.imm = pg.n_rounds + x.a; break;
        case OP_EXPVAL: in.op = X_COIN; in.imm = pg.n_rounds + (uint32_t)n_exposed() + x.a; break;
        case OP_CONST: in.op = X_CONST; in.imm = to_mont(x.a % P); break;
        case OP_ADD:
          if (!ea && !eb) in.op = X_ADD_BB;
          else if (ea && eb) in.op = X_ADD_EE;
          else { in.op = X_ADD_EB; if (!ea) std::swap(ra, rb); }
          break;
        case OP_SUB:
          in.op = (!ea && !eb) ? X_SUB_BB : (ea && eb) ? X_SUB_EE : ea ? X_SUB_EB : X_SUB_BE;
          break;
        default:
          if (!ea && !eb) in.op = X_MUL_BB;
          else if (ea && eb) in.op = X_MUL_EE;
          else { in.op = X_MUL_EB; if (!ea) std::swap(ra, rb); }
      }
      in.a = (uint8_t)ra;
      in.b = (uint8_t)rb;
      reg[id] = (int)d;
      xc.code.push_back(in);
      for (uint32_t r : to_free) free_regs.push_back(r);
    }
    xc.result = (uint32_t)reg[root];
    xc.result_ext = ext_of[root];
    if (xc.n_regs > X_MAX_REGS || xc.code.size() > X_MAX_INST)
      throw Error(LG_ERR_UNSUPPORTED, "constraint expression too large for the device evaluator");
    return xc;
  }

  // ------------------------------------------------------------ setup
  void init_order() {
    exposed.assign(n_exposed(), e6_zero());
    exposed_ready.assign(n_exposed(), 0);
    for (uint32_t m = 0; m < pg.modules.size(); m++) mod_order.push_back(m);
    std::sort(mod_order.begin(), mod_order.end(), [&](uint32_t a, uint32_t b) { return pg.modules[a].name < pg.modules[b].name; });
  }

  // lg_setup (setup/setup.go:68-124): uploads the setup columns (base field,
  // descriptor order), commits the setup tree and keeps tree, LDE, values
  // and coefficients on the context with the program.  Everything allocated
  // here outlives the call.
  void precommit(const uint32_t* const* cols, bool on_device) {
    ArenaScope kept(nullptr);
    init_order();
    size_t total = 0;
    for (const Column& cl : pg.columns)
      if (cl.kind == KIND_SETUP) {
        if (cl.field != 0) throw Error(LG_ERR_UNSUPPORTED, "extension-field setup columns are not supported");
        total += mod_n(cl.module);
      }
    if (!total) throw Error(LG_ERR_INVALID, "the program has no setup columns");
    auto all = std::make_shared<DBuf>(total, c.stream);
    size_t off = 0, si = 0;
    for (uint32_t col = 0; col < pg.columns.size(); col++) {
      const Column& cl = pg.columns[col];
      if (cl.kind != KIND_SETUP) continue;
      const size_t n = mod_n(cl.module);
      if (!cols[si]) throw Error(LG_ERR_INVALID, "null setup column");
      LG_CK(cudaMemcpyAsync(all->p + off, cols[si++], n * 4, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                            c.stream));
      col_buf[col] = dbuf_slice(all, off, n);
      off += n;
    }
    setup_layout();
    auto sd = std::make_shared<SetupData>();
    sd->committed = commit_tree(trees[0]);  // also records the setup columns' coefficients
    sd->root = sd->committed.tree.root;
    for (uint32_t col = 0; col < pg.columns.size(); col++)
      if (pg.columns[col].kind == KIND_SETUP) {
        sd->values[col] = col_buf.at(col);
        sd->coef[col] = col_coef.at(col);
      }
    prog->setup = sd;
  }

  // Host witness: one device buffer for all columns, in column order.  With
  // `split` (lg_prove, tuning upload_split), the columns round 0 commits go
  // up first on the main stream and the others on the side stream right
  // after them, while round 0 runs (await_upload joins them); otherwise
  // every column goes up on the main stream.  Copies of columns that follow
  // one another in host and device memory merge.
  void setup(const uint32_t* const* witness, bool on_device, bool split = false) {
    init_order();
    size_t total_words = 0;
    for (const Column& cl : pg.columns)
      if (cl.kind == KIND_WITNESS) total_words += mod_n(cl.module);
    if (!on_device && total_words) witness_dev = std::make_shared<DBuf>(total_words, c.stream);
    upload_pending = false;
    std::vector<const uint32_t*> src(pg.columns.size(), nullptr);
    size_t wi = 0, woff = 0;
    for (uint32_t col = 0; col < pg.columns.size(); col++) {
      const Column& cl = pg.columns[col];
      size_t n = mod_n(cl.module);
      if (cl.kind == KIND_WITNESS) {
        if (cl.field != 0) throw Error(LG_ERR_UNSUPPORTED, "extension-field witness columns are not supported");
        auto b = std::make_shared<DBuf>();
        b->words = n;
        b->borrowed = true;
        src[col] = witness[wi++];
        if (on_device) {
          // read-only input: use the caller's device buffer as it is
          b->p = const_cast<uint32_t*>(src[col]);
        } else {
          b->p = witness_dev->p + woff;
          woff += n;
        }
        col_buf[col] = b;
      } else if (cl.kind == KIND_LAGRANGE) {
        // 1 at its row: a program constant, kept on the context
        auto key = std::make_pair(pg.modules[cl.module].log_n, lagrange_row(col));
        auto it = c.lagrange_vals.find(key);
        if (it == c.lagrange_vals.end()) {
          ArenaScope kept(nullptr);
          auto b = std::make_shared<DBuf>(n, c.stream);
          LG_CK(cudaMemsetAsync(b->p, 0, n * 4, c.stream));
          uint32_t one = MONT_ONE;
          c.h2d(b->p + key.second, &one, 4);
          it = c.lagrange_vals.emplace(key, b).first;
        }
        col_buf[col] = it->second;
      } else if (cl.kind == KIND_SETUP) {  // precommitted by lg_setup
        if (!prog->setup) throw Error(LG_ERR_INVALID, "the program has setup columns: precommit them with lg_setup first");
        col_buf[col] = prog->setup->values.at(col);
        col_coef[col] = prog->setup->coef.at(col);
      }
    }
    if (!on_device && total_words) {
      // early: the witness columns round 0 commits (all of them unless split)
      std::vector<char> early(pg.columns.size(), 1);
      bool any_late = false;
      if (split && c.tune.upload_split && c.side && c.upload_ev && !pg.staged.empty()) {
        std::fill(early.begin(), early.end(), 0);
        for (uint32_t col : pg.staged[0]) early.at(col) = 1;
        for (uint32_t col = 0; col < pg.columns.size(); col++)
          any_late = any_late || (pg.columns[col].kind == KIND_WITNESS && !early[col]);
        if (!any_late) std::fill(early.begin(), early.end(), 1);
      }
      auto copy = [&](bool want, cudaStream_t s) {
        const uint32_t* run_src = nullptr;
        uint32_t* run_dst = nullptr;
        size_t run_words = 0;
        auto flush = [&]() {
          if (run_words) LG_CK(cudaMemcpyAsync(run_dst, run_src, run_words * 4, cudaMemcpyHostToDevice, s));
          run_words = 0;
        };
        for (uint32_t col = 0; col < pg.columns.size(); col++) {
          if (pg.columns[col].kind != KIND_WITNESS || (early[col] != 0) != want) continue;
          const size_t n = mod_n(pg.columns[col].module);
          uint32_t* dst = col_buf[col]->p;
          if (run_words && src[col] == run_src + run_words && dst == run_dst + run_words) run_words += n;
          else { flush(); run_src = src[col]; run_dst = dst; run_words = n; }
        }
        flush();
      };
      copy(true, c.stream);
      if (any_late) {
        // after the early copies (no contention for the link), on the side
        // stream; the main stream waits for upload_ev before round 1
        LG_CK(cudaEventRecord(c.fork_ev, c.stream));
        LG_CK(cudaStreamWaitEvent(c.side, c.fork_ev, 0));
        copy(false, c.side);
        LG_CK(cudaEventRecord(c.upload_ev, c.side));
        upload_pending = true;
      }
    }
    setup_layout();
  }

  // The main stream waits for the late columns of a split upload.
  void await_upload() {
    if (!upload_pending) return;
    LG_CK(cudaStreamWaitEvent(c.stream, c.upload_ev, 0));
    upload_pending = false;
  }

  // Module order is set; folded relations, degrees, shift schedule and the
  // tree layout (no column data needed).
  void setup_layout() {
    // fold relations with coin(last round) (board/program.go:62-80)
    fold_root.assign(pg.modules.size(), -1);
    degree.assign(pg.modules.size(), NEG_INF);
    root_ext.assign(pg.modules.size(), false);
    for (uint32_t m = 0; m < pg.modules.size(); m++) {
      const auto& rels = pg.modules[m].rels;
      if (rels.empty()) continue;
      uint32_t res = rels.back();
      for (int i = (int)rels.size() - 2; i >= 0; i--) {
        uint32_t cn = push(OP_COIN, pg.n_rounds - 1, 0);
        uint32_t t = push(OP_MUL, cn, res);
        res = push(OP_ADD, rels[i], t);
      }
      fold_root[m] = (int)res;
    }
    compute_ext();
    std::vector<int> memo(pg.nodes.size(), INT32_MIN);  // a node's degree does not depend on the module
    for (uint32_t m = 0; m < pg.modules.size(); m++) {
      if (fold_root[m] < 0) continue;
      degree[m] = node_degree((uint32_t)fold_root[m], memo);
      root_ext[m] = ext_of[fold_root[m]];
    }
    // shift schedule (internal/protocol/schedule.go:92-157)
    std::vector<char> seen(pg.nodes.size(), 0);
    std::vector<uint32_t> reach;
    for (uint32_t m : mod_order) {
      if (fold_root[m] < 0) continue;
      // the nodes under this module's relation only (marks cleared after)
      reach.clear();
      collect((uint32_t)fold_root[m], seen, &reach);
      int64_t n = (int64_t)mod_n(m);
      std::sort(reach.begin(), reach.end());  // node order, as a full scan visits them
      for (uint32_t id : reach) seen[id] = 0;
      for (uint32_t id : reach) {
        if (pg.nodes[id].op != OP_COL) continue;
        const Column& cl = pg.columns[pg.nodes[id].a];
        if (cl.kind == KIND_LAGRANGE) continue;
        int64_t sh = (int32_t)pg.nodes[id].b;
        int s = (int)(((sh % n) + n) % n);
        auto& v = col_shifts[pg.nodes[id].a];
        if (std::find(v.begin(), v.end(), s) == v.end()) v.push_back(s);
      }
    }
    for (auto& kv : col_shifts) std::sort(kv.second.begin(), kv.second.end());
    // layout (internal/protocol/layout.go:165-241): the setup tree (setup
    // columns by module, sorted by name within a module; layout.go:131-151),
    // one tree per round, the AIR tree
    {
      TreeL t{false, -2, {}, true};
      for (uint32_t m : mod_order) {
        std::vector<uint32_t> cols;
        for (uint32_t col = 0; col < pg.columns.size(); col++)
          if (pg.columns[col].kind == KIND_SETUP && pg.columns[col].module == m) cols.push_back(col);
        std::sort(cols.begin(), cols.end(), [&](uint32_t a, uint32_t b) { return pg.columns[a].name < pg.columns[b].name; });
        Group g{m, {}, {}};
        for (uint32_t col : cols) (pg.columns[col].field == 0 ? g.bcols : g.ecols).push_back(col);
        if (!g.bcols.empty() || !g.ecols.empty()) t.groups.push_back(g);
      }
      if (!t.groups.empty()) trees.push_back(t);
    }
    for (uint32_t r = 0; r < pg.n_rounds; r++) {
      TreeL t{false, (int)r, {}};
      for (uint32_t m : mod_order) {
        Group g{m, {}, {}};
        for (uint32_t col : pg.staged[r]) {
          if (pg.columns[col].module != m) continue;
          if (pg.columns[col].kind == KIND_LAGRANGE) throw Error(LG_ERR_INVALID, "verifier column staged for commitment");
          if (pg.columns[col].kind == KIND_SETUP) throw Error(LG_ERR_INVALID, "setup column staged in a round");
          (pg.columns[col].field == 0 ? g.bcols : g.ecols).push_back(col);
        }
        if (!g.bcols.empty() || !g.ecols.empty()) t.groups.push_back(g);
      }
      if (!t.groups.empty()) trees.push_back(t);
    }
    TreeL air{true, -1, {}};
    for (uint32_t m : mod_order) {
      uint32_t nch = chunk_count(m);
      if (!nch) continue;
      Group g{m, {}, {}};
      for (uint32_t k = 0; k < nch; k++) (root_ext[m] ? g.ecols : g.bcols).push_back(k);
      air.groups.push_back(g);
    }
    if (!air.groups.empty()) trees.push_back(air);
    for (uint32_t m = 0; m < pg.modules.size(); m++)
      if (pg.modules[m].log_n > MAX_LOG_MODULE) throw Error(LG_ERR_INVALID, "module above 2^22 rows");
  }

  // row of a Lagrange column (board/module.go:56-82: i, or N-1-i for relative rows)
  uint32_t lagrange_row(uint32_t col) const {
    const Column& cl = pg.columns[col];
    int64_t n = (int64_t)mod_n(cl.module);
    int64_t row = cl.param >= 0 ? cl.param : n - 1 - (-(int64_t)cl.param - 1);
    if (row < 0 || row >= n) throw Error(LG_ERR_INVALID, "Lagrange column row out of range");
    return (uint32_t)row;
  }

  uint32_t chunk_count(uint32_t m) const {
    if (fold_root[m] < 0 || degree[m] <= 0) return 0;
    size_t n = mod_n(m), want = (size_t)std::max(degree[m] - 1, 1) * n, big = 1;
    while (big < want) big <<= 1;
    return (uint32_t)(big / n);
  }

  // Round coins, then per exposed value its average value / N (N: the size of
  // the exposing step's module), then the exposed values themselves, as E6
  // Montgomery words.
  // The kernels' challenge table, assembled on the device from the coin
  // slots and the exposed values (k_coins_assemble): no host round trip, so
  // it works the same whether the coins came from the host transcript or
  // from the device's (fs_slots).
  DBufP coins_on_device() {
    const uint32_t R = pg.n_rounds, X = (uint32_t)n_exposed();
    std::vector<uint32_t> ninv(std::max<uint32_t>(X, 1), 0);
    for (const Step& st : pg.steps)
      if (exposes(st.type) && exposed_ready[st.exposed]) ninv[st.exposed] = inv(to_mont((uint32_t)mod_n(st.module)));
    auto nd = upload_vec(c, ninv);
    const size_t words = 6 * ((size_t)R + 2 * (size_t)X);
    auto out = std::make_shared<DBuf>(std::max<size_t>(words, 1), c.stream);
    if (words) {
      k_coins_assemble<<<(unsigned)((words + 255) / 256), 256, 0, c.stream>>>(
          fs_slots->p, R, exposed_d ? exposed_d->p : nd->p, nd->p, X, out->p);
      LG_LAUNCH();
    }
    return out;
  }

  // ------------------------------------------------------------ steps
  // Grand products of round r (internal/poly/iop_utils.go:170-192,316-323):
  // ratio num/den per row, then a product scan.  Batched: one launch per
  // kernel for all steps of the round; plain: one set of launches per step.
  size_t n_exposed() const {
    size_t k = 0;
    for (const Step& st : pg.steps) k += exposes(st.type);
    return k;
  }

  // Lanes of the columns an expression reads, in first-use order (lane_of
  // for compile_expr).
  struct LaneTable {
    Prover* pr;
    std::vector<const uint32_t*> lanes;
    std::map<uint32_t, uint32_t> first;
    uint32_t operator()(uint32_t col) {
      auto it = first.find(col);
      if (it != first.end()) return it->second;
      if (!pr->col_buf.count(col)) throw Error(LG_ERR_INVALID, "step reads a column that is not available yet");
      uint32_t f = (uint32_t)lanes.size();
      for (uint32_t w = 0; w < pr->lanes_of(col); w++) lanes.push_back(pr->lane_ptr(col, w));
      first[col] = f;
      return f;
    }
  };
  // module whose rows an expression ranges over: that of its first column
  uint32_t expr_module(uint32_t root) {
    std::vector<char> seen(pg.nodes.size(), 0);
    collect(root, seen);
    for (uint32_t i = 0; i < pg.nodes.size(); i++)
      if (seen[i] && pg.nodes[i].op == OP_COL) return pg.columns[pg.nodes[i].a].module;
    throw Error(LG_ERR_INVALID, "lookup table without a column");
  }

  // Lookup multiplicities of width-1 tables, all steps of a round in one set
  // of launches (k_mult_insert / k_mult_count / k_mult_write).
  void run_multiplicities(const std::vector<const Step*>& steps, const DBufP& coins_d) {
    std::vector<DBufP> keep;
    std::vector<EvalJob> evals;
    uint32_t eval_regs = 1, eval_n = 0;
    // device values of one table: the column itself when the expression is
    // a plain unshifted base column, else an evaluation
    auto values = [&](uint32_t root, uint32_t& n) -> const uint32_t* {
      const Node& x = pg.nodes[root];
      uint32_t mod = expr_module(root);
      n = (uint32_t)mod_n(mod);
      if (x.op == OP_COL && x.b == 0 && pg.columns[x.a].field == 0 && col_buf.count(x.a)) return lane_ptr(x.a, 0);
      if (ext_of[root]) throw Error(LG_ERR_INVALID, "lookup table values must be base-field");
      LaneTable lt{this, {}, {}};
      const CodeSet& cs = compiled("e" + std::to_string(root), lt, {root});
      auto tab = upload_vec(c, lt.lanes);
      auto out = std::make_shared<DBuf>(n, c.stream);
      keep.insert(keep.end(), {tab, out});
      evals.push_back(EvalJob{cs.dev[0], (const uint32_t* const*)tab->p, out->p, (int)pg.modules[mod].log_n});
      eval_regs = std::max(eval_regs, cs.xc[0].n_regs);
      eval_n = std::max(eval_n, n);
      return out->p;
    };
    std::vector<MultTab> tabs;
    std::vector<MultVec> tv, sv;
    uint32_t max_t = 1, max_s = 1;
    for (const Step* st : steps) {
      uint32_t tab = (uint32_t)tabs.size(), comb = 0;
      for (size_t k = 0; k < st->tgt.size(); k++) {
        uint32_t n = 0;
        const uint32_t* v = values(st->tgt[k], n);
        uint32_t out = st->outs[k];
        if (pg.columns[out].field != 0 || mod_n(pg.columns[out].module) != n)
          throw Error(LG_ERR_INVALID, "multiplicity column must be a base column of its table's module");
        auto b = std::make_shared<DBuf>(n, c.stream);
        col_buf[out] = b;
        tv.push_back(MultVec{v, n, comb, tab, b->p});
        comb += n;
        max_t = std::max(max_t, n);
      }
      for (uint32_t src : st->src) {
        uint32_t n = 0;
        const uint32_t* v = values(src, n);
        sv.push_back(MultVec{v, n, 0, tab, nullptr});
        max_s = std::max(max_s, n);
      }
      uint32_t cap = 64;
      while (cap < 2 * comb) cap <<= 1;
      auto mem = std::make_shared<DBuf>((size_t)2 * cap + comb, c.stream);
      keep.push_back(mem);
      LG_CK(cudaMemsetAsync(mem->p, 0xff, (size_t)2 * cap * 4, c.stream));
      LG_CK(cudaMemsetAsync(mem->p + 2 * (size_t)cap, 0, (size_t)comb * 4, c.stream));
      tabs.push_back(MultTab{mem->p, mem->p + cap, mem->p + 2 * (size_t)cap, cap});
    }
    auto missing = std::make_shared<DBuf>(1, c.stream);
    LG_CK(cudaMemsetAsync(missing->p, 0, 4, c.stream));
    auto tabs_d = upload_vec(c, tabs), tv_d = upload_vec(c, tv), sv_d = upload_vec(c, sv);
    c.timed("lookup_multiplicities", 0, 0, [&] {
      if (!evals.empty()) {
        auto ed = upload_vec(c, evals);
        keep.push_back(ed);
        const int T = 128;
        size_t smem = (size_t)eval_regs * 6 * T * 4;
        allow_smem(k_eval_base, smem);
        k_eval_base<<<dim3((eval_n + T - 1) / T, (unsigned)evals.size()), T, smem, c.stream>>>(
            (const EvalJob*)ed->p, (const E6*)coins_d->p);
        LG_LAUNCH();
      }
      k_mult_insert<<<dim3((max_t + 255) / 256, (unsigned)tv.size()), 256, 0, c.stream>>>((const MultVec*)tv_d->p,
                                                                                         (const MultTab*)tabs_d->p);
      LG_LAUNCH();
      k_mult_count<<<dim3((max_s + 255) / 256, (unsigned)sv.size()), 256, 0, c.stream>>>(
          (const MultVec*)sv_d->p, (const MultTab*)tabs_d->p, missing->p);
      LG_LAUNCH();
      k_mult_write<<<dim3((max_t + 255) / 256, (unsigned)tv.size()), 256, 0, c.stream>>>((const MultVec*)tv_d->p,
                                                                                        (const MultTab*)tabs_d->p);
      LG_LAUNCH();
    });
    uint32_t* h = c.host_staging(1);
    c.d2h(h, missing->p, 1);
    if (*h) throw Error(LG_ERR_INVALID, "lookup: a source value is not in its table");
  }

  // Lookup multiplicities of tuples with optional selectors, all type-4 steps
  // of a round in one set of launches: target tuples into `keys`, insertion
  // (first selected row per tuple), selected source weights, multiplicity
  // columns (k_tuple_*).
  void run_tuple_multiplicities(const std::vector<const Step*>& steps, const DBufP& coins_d) {
    std::vector<DBufP> keep;
    std::vector<EvalJob> evals;
    uint32_t eval_regs = 1, eval_n = 0;
    auto values = [&](uint32_t root, uint32_t mod) -> const uint32_t* {
      const Node& x = pg.nodes[root];
      const uint32_t n = (uint32_t)mod_n(mod);
      if (expr_module(root) != mod) throw Error(LG_ERR_INVALID, "lookup: a table spans modules");
      if (x.op == OP_COL && x.b == 0 && pg.columns[x.a].field == 0 && col_buf.count(x.a)) return lane_ptr(x.a, 0);
      if (ext_of[root]) throw Error(LG_ERR_INVALID, "lookup tuples and selectors must be base-field");
      LaneTable lt{this, {}, {}};
      const CodeSet& cs = compiled("e" + std::to_string(root), lt, {root});
      auto tab = upload_vec(c, lt.lanes);
      auto out = std::make_shared<DBuf>(n, c.stream);
      keep.insert(keep.end(), {tab, out});
      evals.push_back(EvalJob{cs.dev[0], (const uint32_t* const*)tab->p, out->p, (int)pg.modules[mod].log_n});
      eval_regs = std::max(eval_regs, cs.xc[0].n_regs);
      eval_n = std::max(eval_n, n);
      return out->p;
    };
    std::vector<TupleTab> tabs;
    std::vector<TupleVec> tv, sv;
    uint32_t max_t = 1, max_s = 1;
    for (const Step* st : steps) {
      const uint32_t W = st->width, tab = (uint32_t)tabs.size();
      auto table = [&](const std::vector<uint32_t>& nodes_, size_t k, const std::vector<uint32_t>& sels) {
        TupleVec V{};
        const uint32_t mod = expr_module(nodes_[k * W]);
        V.n = (uint32_t)mod_n(mod);
        for (uint32_t w = 0; w < W; w++) V.comp[w] = values(nodes_[k * W + w], mod);
        V.sel = sels.empty() ? nullptr : values(sels[k], mod);
        V.tab = tab;
        return V;
      };
      uint32_t comb = 0;
      for (size_t k = 0; k < st->outs.size(); k++) {
        TupleVec V = table(st->tgt, k, st->sel_t);
        const uint32_t out = st->outs[k];
        if (pg.columns[out].field != 0 || mod_n(pg.columns[out].module) != V.n)
          throw Error(LG_ERR_INVALID, "multiplicity column must be a base column of its table's module");
        auto b = std::make_shared<DBuf>(V.n, c.stream);
        col_buf[out] = b;
        V.out = b->p;
        V.comb_off = comb;
        comb += V.n;
        max_t = std::max(max_t, V.n);
        tv.push_back(V);
      }
      for (size_t k = 0; k < st->src.size() / W; k++) {
        TupleVec V = table(st->src, k, st->sel_s);
        max_s = std::max(max_s, V.n);
        sv.push_back(V);
      }
      uint32_t cap = 64;
      while (cap < 2 * comb) cap <<= 1;
      auto mem = std::make_shared<DBuf>((size_t)4 * cap + (size_t)comb * W, c.stream);
      keep.push_back(mem);
      LG_CK(cudaMemsetAsync(mem->p, 0xff, (size_t)2 * cap * 4, c.stream));
      LG_CK(cudaMemsetAsync(mem->p + 2 * (size_t)cap, 0, (size_t)2 * cap * 4, c.stream));
      tabs.push_back(TupleTab{mem->p, mem->p + cap, (unsigned long long*)(mem->p + 2 * (size_t)cap),
                              mem->p + 4 * (size_t)cap, cap, W});
    }
    auto flags = std::make_shared<DBuf>(1, c.stream);
    LG_CK(cudaMemsetAsync(flags->p, 0, 4, c.stream));
    auto tabs_d = upload_vec(c, tabs), tv_d = upload_vec(c, tv), sv_d = upload_vec(c, sv);
    c.timed("lookup_multiplicities", 0, 0, [&] {
      if (!evals.empty()) {
        auto ed = upload_vec(c, evals);
        keep.push_back(ed);
        const int T = 128;
        size_t smem = (size_t)eval_regs * 6 * T * 4;
        allow_smem(k_eval_base, smem);
        k_eval_base<<<dim3((eval_n + T - 1) / T, (unsigned)evals.size()), T, smem, c.stream>>>(
            (const EvalJob*)ed->p, (const E6*)coins_d->p);
        LG_LAUNCH();
      }
      const dim3 gt((max_t + 255) / 256, (unsigned)tv.size()), gs((max_s + 255) / 256, (unsigned)sv.size());
      k_tuple_keys<<<gt, 256, 0, c.stream>>>((const TupleVec*)tv_d->p, (const TupleTab*)tabs_d->p);
      LG_LAUNCH();
      k_tuple_insert<<<gt, 256, 0, c.stream>>>((const TupleVec*)tv_d->p, (const TupleTab*)tabs_d->p, flags->p);
      LG_LAUNCH();
      k_tuple_count<<<gs, 256, 0, c.stream>>>((const TupleVec*)sv_d->p, (const TupleTab*)tabs_d->p, flags->p);
      LG_LAUNCH();
      k_tuple_write<<<gt, 256, 0, c.stream>>>((const TupleVec*)tv_d->p, (const TupleTab*)tabs_d->p);
      LG_LAUNCH();
    });
    uint32_t* h = c.host_staging(1);
    c.d2h(h, flags->p, 1);
    if (*h & 2) throw Error(LG_ERR_INVALID, "lookup: hash table full");
    if (*h & 1) throw Error(LG_ERR_INVALID, "lookup: a source value is not in its table");
  }

  // Cyclic logup columns and their totals (board/logup.go:129-180): one set of
  // launches over all logup steps of a round (batched) or one per step.
  void run_logups(const std::vector<const Step*>& steps, const DBufP& coins_d) {
    std::vector<DBufP> keep;
    std::vector<LogupJob> jobs;
    std::vector<ScanJob> scans;
    std::vector<LogupFinish> fins;
    uint32_t max_regs = 1;
    for (const Step* st : steps) {
      if (st->e.size() > (size_t)LOGUP_MAX_TERMS)
        throw Error(LG_ERR_UNSUPPORTED, "logup columns of more than 4 fractions are not supported by this build");
      if (pg.columns[st->out].field != 1 || pg.columns[st->out].module != st->module)
        throw Error(LG_ERR_INVALID, "logup column must be an extension column of its module");
      uint32_t logn = pg.modules[st->module].log_n;
      size_t n = (size_t)1 << logn;
      LaneTable lt{this, {}, {}};
      LogupJob J{};
      J.n_terms = (uint32_t)st->e.size();
      std::vector<uint32_t> roots;
      for (size_t k = 0; k < st->e.size(); k++) { roots.push_back(st->e[k]); roots.push_back(st->m[k]); }
      const CodeSet& cs = compiled("l" + std::to_string(step_index(st)), lt, roots);
      for (size_t k = 0; k < st->e.size(); k++) {
        J.e[k] = cs.dev[2 * k];
        J.m[k] = cs.dev[2 * k + 1];
        max_regs = std::max(max_regs, std::max(cs.xc[2 * k].n_regs, cs.xc[2 * k + 1].n_regs));
      }
      auto tab = upload_vec(c, lt.lanes);
      auto frac = std::make_shared<DBuf>(6 * n, c.stream);
      uint32_t nt = (uint32_t)((n + SCAN_TILE - 1) / SCAN_TILE);
      auto totals = std::make_shared<DBuf>(6 * (size_t)nt, c.stream), pre = std::make_shared<DBuf>(6 * (size_t)nt, c.stream);
      auto res = std::make_shared<DBuf>(6 * n, c.stream);
      keep.insert(keep.end(), {tab, frac, totals, pre});
      J.lanes = (const uint32_t* const*)tab->p;
      J.frac = frac->p;
      J.logn = (int)logn;
      jobs.push_back(J);
      scans.push_back(ScanJob{frac->p, n, totals->p, pre->p, res->p, nt});
      fins.push_back(LogupFinish{exposed_d->p + 6 * (size_t)st->exposed, inv(to_mont((uint32_t)n))});
      col_buf[st->out] = res;
    }
    const int T = 128;
    size_t smem = (size_t)max_regs * 6 * T * 4;
    allow_smem(k_logup_frac, smem);
    auto launch = [&](size_t first, size_t count) {
      uint32_t max_n = 0, max_nt = 0;
      for (size_t i = first; i < first + count; i++) {
        max_n = std::max<uint32_t>(max_n, (uint32_t)scans[i].n);
        max_nt = std::max(max_nt, scans[i].nt);
      }
      std::vector<LogupJob> jv(jobs.begin() + first, jobs.begin() + first + count);
      std::vector<ScanJob> sv(scans.begin() + first, scans.begin() + first + count);
      std::vector<LogupFinish> fv(fins.begin() + first, fins.begin() + first + count);
      auto jd = upload_vec(c, jv), sd = upload_vec(c, sv), fd = upload_vec(c, fv);
      c.timed("logup", 0, 0, [&] {
        k_logup_frac<<<dim3((max_n + T - 1) / T, (unsigned)count), T, smem, c.stream>>>((const LogupJob*)jd->p,
                                                                                        (const E6*)coins_d->p);
        LG_LAUNCH();
        k_scan_tiles<true><<<dim3(max_nt, (unsigned)count), SCAN_BLOCK, 0, c.stream>>>((const ScanJob*)sd->p);
        LG_LAUNCH();
        k_tile_prefix<true><<<(unsigned)((count + 63) / 64), 64, 0, c.stream>>>((const ScanJob*)sd->p, (uint32_t)count);
        LG_LAUNCH();
        k_logup_finish<<<dim3((max_n + 255) / 256, (unsigned)count), 256, 0, c.stream>>>((const ScanJob*)sd->p,
                                                                                         (const LogupFinish*)fd->p);
        LG_LAUNCH();
      });
    };
    if (c.batched) launch(0, jobs.size());
    else for (size_t i = 0; i < jobs.size(); i++) launch(i, 1);
  }

  // Exposed values of round r's steps: read back (Montgomery E6).
  void read_exposed(uint32_t r) {
    std::vector<const Step*> lg;
    for (const Step& st : pg.steps) if (st.round == r && exposes(st.type)) lg.push_back(&st);
    if (lg.empty()) return;
    uint32_t* h = c.host_staging(6 * exposed.size());
    c.d2h(h, exposed_d->p, 6 * exposed.size());
    for (const Step* st : lg) {
      for (int w = 0; w < 6; w++) exposed[st->exposed].c[w] = h[6 * st->exposed + w];
      exposed_ready[st->exposed] = 1;
    }
  }

  void run_steps(uint32_t r) {
    std::vector<const Step*> steps, gps, mults, tmults, logups;
    for (const Step& st : pg.steps) {
      if (st.round != r) continue;
      steps.push_back(&st);
      (st.type == STEP_GP || st.type == STEP_RATIO ? gps
       : st.type == STEP_MULT                      ? mults
       : st.type == STEP_MULTW                     ? tmults
                                                   : logups).push_back(&st);
    }
    if (!exposed_d && n_exposed()) exposed_d = std::make_shared<DBuf>(6 * n_exposed(), c.stream);
    if (steps.empty()) return;
    auto coins_d = coins_on_device();
    // steps of one round read only earlier rounds' columns; multiplicities,
    // grand products and logups are independent of each other
    if (!mults.empty()) run_multiplicities(mults, coins_d);
    if (!tmults.empty()) run_tuple_multiplicities(tmults, coins_d);
    if (!logups.empty()) run_logups(logups, coins_d);
    steps = gps;
    if (steps.empty()) return;
    std::vector<GpJob> jobs;
    std::vector<ScanJob> scans;
    std::vector<DBufP> keep;
    std::vector<const uint32_t*> all_lanes;  // every step's lane table, one upload
    std::vector<size_t> lane_off;
    uint32_t max_regs = 1;
    std::vector<const CodeSet*> codes;  // per job: numerator and denominator bytecode
    for (const Step* st : steps) {
      uint32_t logn = pg.modules[st->module].log_n;
      size_t n = (size_t)1 << logn;
      std::vector<const uint32_t*> lanes;
      std::map<uint32_t, uint32_t> first_lane;
      auto lane_of = [&](uint32_t col) -> uint32_t {
        auto it = first_lane.find(col);
        if (it != first_lane.end()) return it->second;
        if (!col_buf.count(col)) throw Error(LG_ERR_INVALID, "step reads a column that is not available yet");
        uint32_t f = (uint32_t)lanes.size();
        for (uint32_t w = 0; w < lanes_of(col); w++) lanes.push_back(lane_ptr(col, w));
        first_lane[col] = f;
        return f;
      };
      const CodeSet& cs = compiled("g" + std::to_string(step_index(st)), lane_of, {st->num, st->den});
      max_regs = std::max(max_regs, std::max(cs.xc[0].n_regs, cs.xc[1].n_regs));
      lane_off.push_back(all_lanes.size());
      all_lanes.insert(all_lanes.end(), lanes.begin(), lanes.end());
      auto ratio = std::make_shared<DBuf>(6 * n, c.stream);
      uint32_t nt = (uint32_t)((n + SCAN_TILE - 1) / SCAN_TILE);
      auto totals = std::make_shared<DBuf>(6 * (size_t)nt, c.stream), pre = std::make_shared<DBuf>(6 * (size_t)nt, c.stream);
      auto res = std::make_shared<DBuf>(6 * n, c.stream);
      keep.insert(keep.end(), {ratio, totals, pre});
      jobs.push_back(GpJob{cs.dev[0], cs.dev[1], nullptr, ratio->p, (int)logn});
      codes.push_back(&cs);
      ScanJob sj{ratio->p, n, totals->p, pre->p, res->p, nt};
      if (st->type == STEP_RATIO) {  // inclusive products; the end is exposed
        if (pg.columns[st->out].field != 1 || pg.columns[st->out].module != st->module)
          throw Error(LG_ERR_INVALID, "running ratio column must be an extension column of its module");
        sj.inclusive = 1;
        sj.end = exposed_d->p + 6 * (size_t)st->exposed;
      }
      scans.push_back(sj);
      col_buf[st->out] = res;
    }
    auto tab_all = upload_vec(c, all_lanes);
    keep.push_back(tab_all);
    for (size_t i = 0; i < jobs.size(); i++) jobs[i].lanes = (const uint32_t* const*)tab_all->p + lane_off[i];
    const int T = 128;
    size_t smem = (size_t)max_regs * 6 * T * 4;
    allow_smem(k_gp_ratio, smem);
    auto launch = [&](size_t first, size_t count) {
      uint32_t max_n = 0, max_nt = 0;
      for (size_t i = first; i < first + count; i++) {
        max_n = std::max<uint32_t>(max_n, (uint32_t)scans[i].n);
        max_nt = std::max(max_nt, scans[i].nt);
      }
      // ratios: compiled kernels per distinct (numerator, denominator)
      // program (xjit.cuh), the interpreter for the rest
      std::vector<GpJob> jv;
      std::map<CUfunction, std::pair<std::vector<GpxJob>, uint32_t>> jit;  // jobs, largest n
      uint32_t max_ni = 0;
      for (size_t i = first; i < first + count; i++) {
        const uint32_t ni = (uint32_t)scans[i].n;
        if (CUfunction f = c.tune.quotient_jit ? jit_of(*codes[i], true) : nullptr) {
          auto& g = jit[f];
          g.first.push_back(GpxJob{jobs[i].lanes, jobs[i].ratio, jobs[i].logn});
          g.second = std::max(g.second, ni);
        } else {
          jv.push_back(jobs[i]);
          max_ni = std::max(max_ni, ni);
        }
      }
      std::vector<ScanJob> sv(scans.begin() + first, scans.begin() + first + count);
      std::vector<std::pair<CUfunction, DBufP>> jit_d;
      for (auto& kv : jit) jit_d.push_back({kv.first, upload_vec(c, kv.second.first)});
      DBufP jd = jv.empty() ? DBufP() : upload_vec(c, jv);
      auto sd = upload_vec(c, sv);
      c.timed("grand_product", 0, 0, [&] {
        for (auto& fd : jit_d) {
          const auto& g = jit.at(fd.first);
          xjit_launch(fd.first, dim3((g.second + 127) / 128, (unsigned)g.first.size()), fd.second->p,
                      (const E6*)coins_d->p, c.stream);
          g_launches.fetch_add(1);
        }
        if (!jv.empty()) {
          k_gp_ratio<<<dim3((max_ni + T - 1) / T, (unsigned)jv.size()), T, smem, c.stream>>>((const GpJob*)jd->p,
                                                                                            (const E6*)coins_d->p);
          LG_LAUNCH();
        }
        k_scan_tiles<<<dim3(max_nt, (unsigned)count), SCAN_BLOCK, 0, c.stream>>>((const ScanJob*)sd->p);
        LG_LAUNCH();
        k_tile_prefix<<<(unsigned)((count + 63) / 64), 64, 0, c.stream>>>((const ScanJob*)sd->p, (uint32_t)count);
        LG_LAUNCH();
        k_gp_finish<<<dim3((max_n + 255) / 256, (unsigned)count), 256, 0, c.stream>>>((const ScanJob*)sd->p);
        LG_LAUNCH();
      });
    };
    if (c.batched) launch(0, jobs.size());
    else for (size_t i = 0; i < jobs.size(); i++) launch(i, 1);
  }

  // ------------------------------------------------------------ commits
  Committed commit_tree(const TreeL& t, bool read_root = true) {
    std::vector<GroupSpec> gs;
    for (const Group& g : t.groups) {
      GroupSpec s;
      s.log_n = pg.modules[g.module].log_n;
      s.nb = (uint32_t)g.bcols.size();
      s.ne = (uint32_t)g.ecols.size();
      size_t n = mod_n(g.module);
      if (t.air) {
        s.from_coeffs = true;
        uint32_t lw = root_ext[g.module] ? 6 : 1;
        const uint32_t* base = chunk_coef.at(g.module)->p;
        for (uint32_t k : g.bcols) s.lanes.push_back(base + (size_t)k * n);
        for (uint32_t k : g.ecols) for (uint32_t w = 0; w < 6; w++) s.lanes.push_back(base + ((size_t)k * lw + w) * n);
      } else {
        s.from_coeffs = false;
        for (uint32_t col : g.bcols) s.lanes.push_back(lane_ptr(col, 0));
        for (uint32_t col : g.ecols) for (uint32_t w = 0; w < 6; w++) s.lanes.push_back(lane_ptr(col, w));
      }
      gs.push_back(s);
    }
    Committed cm = commit(c, gs, !t.air, read_root);
    if (!t.air) {
      for (size_t gi = 0; gi < t.groups.size(); gi++) {
        const Group& g = t.groups[gi];
        size_t n = mod_n(g.module);
        uint32_t lane = 0;
        for (uint32_t col : g.bcols) col_coef[col] = cm.groups[gi].coef->p + (size_t)(lane++) * n;
        for (uint32_t col : g.ecols) { col_coef[col] = cm.groups[gi].coef->p + (size_t)lane * n; lane += 6; }
      }
    }
    return cm;
  }

  // ------------------------------------------------------------ quotient
  // Q = V / (X^N - 1) of every module (internal/poly/compute_quotient.go:223-424),
  // as chunk coefficients: coefficient lanes -> values on the four cosets
  // g w_4n^c <w_n> -> bytecode evaluation and division -> per-coset inverse
  // transforms -> a 4-point inverse DFT across cosets (k_quotient_chunks).
  void quotient_all() {
    struct ModQ {
      uint32_t m, logn;
      std::vector<const uint32_t*> coef_lanes;
      std::vector<CosetLane> lanes;
      DBufP cv, qv, chunks;
      const CodeSet* cs;
      XProgram prog;
      uint32_t zinv[4];
    };
    std::vector<ModQ> mods;
    std::vector<DBufP> keep;
    // log n -> columns -> lanes (Lagrange values -> coefficients)
    std::map<uint32_t, std::vector<std::vector<uint32_t*>>> verifier_intt;
    // Lagrange coefficients first computed by this prove: kept on the context
    // once their transforms are enqueued
    std::map<std::pair<uint32_t, uint32_t>, DBufP> new_lagrange;
    for (uint32_t m : mod_order) {
      if (!chunk_count(m)) continue;
      // Four cosets give all four chunks of Q; a module of lower degree commits
      // the first chunk_count of them (the others vanish for a valid witness).
      if (chunk_count(m) != 1 && chunk_count(m) != 2 && chunk_count(m) != 4)
        throw Error(LG_ERR_UNSUPPORTED, "quotients of more than four chunks are not supported by this build");
      uint32_t logn = pg.modules[m].log_n;
      check_ntt_size((int)logn);
      size_t n = (size_t)1 << logn;
      ModQ q;
      q.m = m;
      q.logn = logn;
      std::vector<const uint32_t*> coef_lanes;
      std::map<uint32_t, uint32_t> first_lane;
      auto lane_of = [&](uint32_t col) -> uint32_t {
        auto it = first_lane.find(col);
        if (it != first_lane.end()) return it->second;
        uint32_t f = (uint32_t)coef_lanes.size();
        auto cc = col_coef.find(col);
        if (cc != col_coef.end()) {
          for (uint32_t w = 0; w < lanes_of(col); w++) coef_lanes.push_back(cc->second + (size_t)w * n);
        } else if (pg.columns[col].kind == KIND_LAGRANGE) {
          // a program constant: coefficients kept from an earlier prove, or
          // computed by this one (values copied, transformed below)
          auto key = std::make_pair(logn, lagrange_row(col));
          auto hit = c.lagrange_coef.find(key);
          DBufP b = hit != c.lagrange_coef.end() ? hit->second : nullptr;
          if (!b && new_lagrange.count(key)) b = new_lagrange.at(key);
          if (!b) {
            ArenaScope kept(nullptr);
            b = std::make_shared<DBuf>(n, c.stream);
            LG_CK(cudaMemcpyAsync(b->p, col_buf.at(col)->p, n * 4, cudaMemcpyDeviceToDevice, c.stream));
            verifier_intt[logn].push_back({b->p});
            new_lagrange[key] = b;
          }
          coef_lanes.push_back(b->p);
        } else {
          // verifier columns: coefficients of the Lagrange values
          auto b = std::make_shared<DBuf>(lanes_of(col) * n, c.stream);
          LG_CK(cudaMemcpyAsync(b->p, col_buf.at(col)->p, lanes_of(col) * n * 4, cudaMemcpyDeviceToDevice, c.stream));
          // transformed in place below: batched, one launch per size over all
          // modules; plain, one launch per column
          std::vector<uint32_t*> ls;
          for (uint32_t w = 0; w < lanes_of(col); w++) ls.push_back(b->p + (size_t)w * n);
          verifier_intt[logn].push_back(ls);
          keep.push_back(b);
          for (uint32_t w = 0; w < lanes_of(col); w++) coef_lanes.push_back(b->p + (size_t)w * n);
        }
        first_lane[col] = f;
        return f;
      };
      const CodeSet& cs = compiled("q" + std::to_string(m), lane_of, {(uint32_t)fold_root[m]});
      q.cs = &cs;
      q.prog = cs.dev[0];
      q.coef_lanes = coef_lanes;
      uint32_t g = to_mont(3), w4n = root_of_unity_mont((int)logn + RATE_LOG);
      for (int cc = 0; cc < 4; cc++) q.zinv[cc] = inv(sub(mont_pow(mul(g, mont_pow(w4n, cc)), n), MONT_ONE));
      mods.push_back(std::move(q));
    }
    {  // coset values, quotient values and chunks of all modules: one allocation each
      size_t cv_words = 0, qv_words = 0, ch_words = 0;
      for (auto& q : mods) {
        const size_t n = (size_t)1 << q.logn, big = n << RATE_LOG, w = root_ext[q.m] ? 6 : 1;
        cv_words += q.coef_lanes.size() * big;
        qv_words += w * big;
        ch_words += 4 * w * n;
      }
      auto cv_all = std::make_shared<DBuf>(cv_words, c.stream);
      auto qv_all = std::make_shared<DBuf>(qv_words, c.stream);
      auto ch_all = std::make_shared<DBuf>(ch_words, c.stream);
      size_t cv_off = 0, qv_off = 0, ch_off = 0;
      for (auto& q : mods) {
        const size_t n = (size_t)1 << q.logn, big = n << RATE_LOG, w = root_ext[q.m] ? 6 : 1;
        q.cv = dbuf_slice(cv_all, cv_off, q.coef_lanes.size() * big);
        cv_off += q.coef_lanes.size() * big;
        for (size_t l = 0; l < q.coef_lanes.size(); l++) q.lanes.push_back(CosetLane{q.coef_lanes[l], q.cv->p + l * big});
        q.qv = dbuf_slice(qv_all, qv_off, w * big);
        qv_off += w * big;
        q.chunks = dbuf_slice(ch_all, ch_off, 4 * w * n);
        ch_off += 4 * w * n;
        chunk_coef[q.m] = q.chunks;
      }
    }
    auto intt_lanes = [&](uint32_t logn, const std::vector<uint32_t*>& lanes) {
      const size_t n = (size_t)1 << logn;
      if ((int)logn > SMEM_NTT_MAX_LOG) {
        std::vector<BigNtt> jobs;
        for (uint32_t* l : lanes) jobs.push_back(big_job(l, l, inv(to_mont((uint32_t)n)), false));
        big_ntt(c, jobs, (int)logn, true, "quotient_intt", 8.0 * n);
        return;
      }
      auto tab = upload_vec(c, lanes);
      keep.push_back(tab);
      const uint32_t* twn = c.ntt_twiddles((int)logn);
      with_ntt_size((int)logn, [&](auto L) {
        allow_smem(k_intt<decltype(L)::value>, pad16_words((int)logn) * 4);
        c.timed("quotient_intt", 8.0 * n * lanes.size(), 0, [&] {
          k_intt<decltype(L)::value><<<(unsigned)lanes.size(), ntt_threads((int)logn), pad16_words((int)logn) * 4,
                                       c.stream>>>((uint32_t* const*)tab->p, (int)logn, twn, inv(to_mont((uint32_t)n)));
          LG_LAUNCH();
        });
      });
    };
    for (auto& kv : verifier_intt) {
      if (c.batched) {
        std::vector<uint32_t*> all;
        for (auto& col : kv.second) all.insert(all.end(), col.begin(), col.end());
        intt_lanes(kv.first, all);
      } else {
        for (auto& col : kv.second) intt_lanes(kv.first, col);
      }
    }
    for (auto& kv : new_lagrange) c.lagrange_coef[kv.first] = kv.second;
    if (mods.empty()) return;
    auto coins_d = coins_on_device();
    const int T = 128;
    auto run = [&](const std::vector<ModQ*>& ms) {
      // 1. coset evaluations, one launch per size
      std::map<uint32_t, std::vector<CosetLane>> by_size;
      for (ModQ* q : ms) by_size[q->logn].insert(by_size[q->logn].end(), q->lanes.begin(), q->lanes.end());
      for (auto& kv : by_size) {
        uint32_t logn = kv.first;
        size_t n = (size_t)1 << logn;
        if ((int)logn > SMEM_NTT_MAX_LOG) {
          std::vector<BigNtt> jobs;
          const uint32_t* tw4 = c.twiddles((int)logn + RATE_LOG);
          const uint32_t* gp = c.gpowers((int)logn, false);
          for (auto& L : kv.second)
            for (int cc = 0; cc < 4; cc++) {
              BigNtt j = big_job(L.src, L.out + (size_t)cc * n, MONT_ONE, false);
              j.t1 = gp;
              j.t2 = tw4;
              j.m2_mask = (uint32_t)((n << RATE_LOG) - 1);
              j.e2 = (uint32_t)cc;
              jobs.push_back(j);
            }
          big_ntt(c, jobs, (int)logn, false, "coset_eval", 5.0 * n);
          continue;
        }
        auto tab = upload_vec(c, kv.second);
        const uint32_t* twn = c.ntt_twiddles((int)logn);
        const uint32_t* shifts = c.coset_shifts((int)logn);
        const size_t smem = 2 * pad16_words((int)logn) * 4;
        with_ntt_size((int)logn, [&](auto L) {
          allow_smem(k_coset_eval<decltype(L)::value>, smem);
          c.timed("coset_eval", 20.0 * n * kv.second.size(), 0, [&] {
            k_coset_eval<decltype(L)::value><<<dim3((unsigned)kv.second.size(), 4), ntt_threads((int)logn), smem,
                                               c.stream>>>((const CosetLane*)tab->p, (int)logn, twn, shifts);
            LG_LAUNCH();
          });
        });
      }
      // 2. bytecode evaluation on the 4n coset points of every module
      // modules whose bytecode compiles to a kernel of its own (xjit.cuh) run
      // it, one launch per distinct program; the others the interpreter
      std::vector<QJob> qj;
      std::map<CUfunction, std::pair<std::vector<QxJob>, uint32_t>> jit;  // jobs, largest n
      uint32_t max_regs = 1, max_n = 0;
      double qbytes = 0;
      for (ModQ* q : ms) {
        qbytes += (4.0 * q->lanes.size() + 24.0) * (4.0 * (1u << q->logn));
        max_n = std::max(max_n, 1u << q->logn);  // the chunk step below covers every module
        if (CUfunction f = c.tune.quotient_jit ? jit_of(*q->cs, false) : nullptr) {
          QxJob x{q->cv->p, q->qv->p, (int)q->logn, {q->zinv[0], q->zinv[1], q->zinv[2], q->zinv[3]}};
          auto& g = jit[f];
          g.first.push_back(x);
          g.second = std::max(g.second, 1u << q->logn);
          continue;
        }
        QJob j{};
        j.p = q->prog;
        j.cv = q->cv->p;
        j.qv = q->qv->p;
        j.logn = (int)q->logn;
        for (int k = 0; k < 4; k++) j.zinv[k] = q->zinv[k];
        qj.push_back(j);
        max_regs = std::max(max_regs, q->cs->xc[0].n_regs);
      }
      std::vector<std::pair<CUfunction, DBufP>> jit_d;
      for (auto& kv : jit) jit_d.push_back({kv.first, upload_vec(c, kv.second.first)});
      DBufP qd = qj.empty() ? DBufP() : upload_vec(c, qj);
      size_t smem = (size_t)max_regs * 6 * T * 4;
      if (!qj.empty()) allow_smem(k_quotient_eval, smem);
      c.timed("quotient_eval", qbytes, 0, [&] {
        for (auto& fd : jit_d) {
          const auto& g = jit.at(fd.first);
          xjit_launch(fd.first, dim3((g.second + 127) / 128, 4, (unsigned)g.first.size()), (const QxJob*)fd.second->p,
                      (const E6*)coins_d->p, c.stream);
          g_launches.fetch_add(1);
        }
        if (!qj.empty()) {
          k_quotient_eval<<<dim3((max_n + T - 1) / T, 4, (unsigned)qj.size()), T, smem, c.stream>>>(
              (const QJob*)qd->p, (const E6*)coins_d->p);
          LG_LAUNCH();
        }
      });
      // 3. per-coset inverse transforms, one launch per size
      std::map<uint32_t, std::vector<uint32_t*>> intt;
      for (ModQ* q : ms) {
        size_t n = (size_t)1 << q->logn;
        uint32_t lw = root_ext[q->m] ? 6 : 1;
        for (uint32_t w = 0; w < lw; w++)
          for (int cc = 0; cc < 4; cc++) intt[q->logn].push_back(q->qv->p + (size_t)w * 4 * n + cc * n);
      }
      for (auto& kv : intt) {
        size_t n = (size_t)1 << kv.first;
        if ((int)kv.first > SMEM_NTT_MAX_LOG) {
          std::vector<BigNtt> jobs;
          for (uint32_t* l : kv.second) jobs.push_back(big_job(l, l, inv(to_mont((uint32_t)n)), false));
          big_ntt(c, jobs, (int)kv.first, true, "quotient_intt", 8.0 * n);
          continue;
        }
        auto tab = upload_vec(c, kv.second);
        const uint32_t* twn = c.ntt_twiddles((int)kv.first);
        with_ntt_size((int)kv.first, [&](auto L) {
          allow_smem(k_intt<decltype(L)::value>, pad16_words((int)kv.first) * 4);
          c.timed("quotient_intt", 8.0 * n * kv.second.size(), 0, [&] {
            k_intt<decltype(L)::value><<<(unsigned)kv.second.size(), ntt_threads((int)kv.first),
                                         pad16_words((int)kv.first) * 4, c.stream>>>(
                (uint32_t* const*)tab->p, (int)kv.first, twn, inv(to_mont((uint32_t)n)));
            LG_LAUNCH();
          });
        });
      }
      // 4. chunk coefficients
      std::vector<QcJob> cj;
      for (ModQ* q : ms) {
        size_t n = (size_t)1 << q->logn;
        cj.push_back(QcJob{q->qv->p, q->chunks->p, (int)q->logn, root_ext[q->m] ? 6u : 1u,
                           c.gpowers((int)q->logn, true), c.twiddles((int)q->logn + RATE_LOG),
                           inv(mont_pow(to_mont(3), n))});
      }
      auto cd = upload_vec(c, cj);
      c.timed("quotient_chunks", 0, 0, [&] {
        k_quotient_chunks<<<dim3((max_n + 127) / 128, 6, (unsigned)cj.size()), 128, 0, c.stream>>>(
            (const QcJob*)cd->p, inv(to_mont(4)));
        LG_LAUNCH();
      });
    };
    if (c.batched) {
      std::vector<ModQ*> all;
      for (auto& q : mods) all.push_back(&q);
      run(all);
    } else {
      for (auto& q : mods) run({&q});
    }
  }

  // ------------------------------------------------------------ phases
  // The prove as a sequence of device phases (prove_flow.cuh).  Each phase
  // needs the challenges that the transcript derives from the results of the
  // phases before it; the caller keeps the transcript (lg_prove: the host
  // Transcript below; the session entry points: the caller of the C ABI)
  // and hands the challenges in with set_challenge.
  void begin(const uint32_t* const* witness, bool on_device, bool split_upload = false);
  bool has_setup_tree() const { return !trees.empty() && trees[0].setup; }
  // ExecuteSteps + commitTraceRound of round r (prover/prover.go:321-411):
  // true with the root when the round commits a tree.
  bool commit_round(uint32_t r, Digest* root);
  // the exposed values of round r's steps, in step order (Montgomery E6)
  std::vector<E6> round_exposed(uint32_t r) const;
  // ComputeAIRQuotients and the AIR commitment (prover/prover.go:461-561)
  bool commit_quotient(Digest* root);
  // claimed values at zeta (internal/fri/values.go:46-110), and the order
  // bindClaimedValuesByPolynomialOrder binds them (internal/fri/open.go:223-285)
  void claimed_values();
  std::vector<E6> claimed_values_bind_order() const;
  // DEEP classes (modules with committed groups, layout order) and, per
  // class, its opening points as the factors w_n^shift of z = zeta w_n^shift
  // in first-use order (the order k_deep's points take)
  std::vector<uint32_t> deep_class_list() const;
  std::vector<uint32_t> class_point_factors(uint32_t m) const;
  // k_deep_den for every class on the side stream (needs zeta in its slot)
  void launch_deep_den();
  void deep_codewords();                  // internal/fri/deep.go:71-266
  Digest commit_levels();                 // fri.Prove's levels tree (internal/fri/fri.go:294-317)
  // fold round j (foldLayerExt) with the challenge at chal + 8 j, then the
  // next layer's commitment; true with its root (read back when read_root)
  // next_fs: hash the next fold challenge with the new tree's top when that
  // runs as one block (*fused says whether it did)
  bool fri_fold_round(int j, bool read_root, Digest* next_root, const FsTail* next_fs = nullptr,
                      bool* fused = nullptr);
  void read_final_poly();
  // rounds j0 .. NR - 1 in one block (k_fri_tail), challenge j0 already on
  // the device; the same layers, trees and challenges as fri_fold_round
  void fri_tail(int j0, const DBufP& pre_d, const std::vector<uint32_t>& pre_off, const std::vector<uint32_t>& pre_len);
  // query openings at positions (openQueryExt, openCommittedAt) and the
  // canonical encoding of the whole proof
  size_t open_and_encode(const std::vector<uint32_t>& pos, uint8_t* out, size_t out_cap, bool* in_out);
  void plan_openings();
  // challenge by its transcript name: challenge@loom_<r> and __zeta (E6 from
  // the digest's first six words), alpha_DEEP, fri_level_<l>_gamma,
  // fri_fold_<j> (the whole digest)
  void set_challenge(const std::string& name, const uint32_t* digest);
  // Device transcript (dev_fs): appends challenge `name` to q — the words
  // the host transcript already has for it, the previous challenge's digest
  // from prev_dev when the host does not have it yet, then `dev` (device
  // words, in order) — with its digest going to `out`; false when the
  // message is longer than k_fs_chain takes.
  bool fs_queue(FsQueue& q, const std::string& name, const uint32_t* prev_dev, const DevWords& dev, uint32_t* out);
  void fs_launch(FsQueue& q);
  // Reads back the pending roots, the exposed values and the coin and zeta
  // slots, and replays the pending challenges on the host transcript; each
  // digest must equal the device's.
  void sync_transcript();
  void need_coins(uint32_t r) const {
    for (uint32_t k = 0; k < r; k++)
      if (!coin_ready[k]) throw Error(LG_ERR_INVALID, "challenge " + coin_name(k) + " has not been set");
  }

  // Whole prove with the host transcript (lg_prove).  Returns the proof
  // length.  The bytes go to out[0, out_cap) when they fit (*in_out = true),
  // else to c.proof_buf.
  size_t prove(const uint32_t* const* witness, bool on_device, uint8_t* out, size_t out_cap, bool* in_out);
};

}  // namespace lg
