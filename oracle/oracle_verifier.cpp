// CPU oracle (test infrastructure): verifier of the canonical proof encoding
// for the Poseidon2 backend.  It restates loom's acceptance checks:
//  * transcript replay, claimed values, verifier columns and the AIR relation
//    at zeta: verifier/verifier.go:119-533, verifier/hookFns.go:34-97;
//  * alpha_DEEP replay, Merkle openings with injections and the DEEP bridge:
//    internal/fri/verify.go:60-700;
//  * multi-degree FRI query checks: internal/fri/fri.go:751-1022,1430-1530;
//  * paths with injections: internal/merkle/tree.go:392-436.
// The program layout (module order, folded relations, shift schedule, trees,
// chunk counts) comes from the prover's own setup_layout, so a proof is
// checked against the same schedule it was produced under; everything else
// (transcript, hashing, arithmetic at zeta, FRI) is recomputed here from the
// proof bytes alone.
#include "prover_core.h"

namespace orc {
namespace {

// ------------------------------------------------------------ proof decoding
struct Reader {
  const uint8_t* b;
  size_t n, pos = 0;
  uint32_t u32() {
    if (n - pos < 4) throw std::runtime_error("proof: truncated");
    uint32_t x = ((uint32_t)b[pos] << 24) | ((uint32_t)b[pos + 1] << 16) | ((uint32_t)b[pos + 2] << 8) | (uint32_t)b[pos + 3];
    pos += 4;
    return x;
  }
  uint32_t el() {
    uint32_t x = u32();
    if (x >= P) throw std::runtime_error("proof: field element not reduced");
    return x;
  }
  E6 e6() { E6 r; for (int i = 0; i < 6; i++) r.c[i] = el(); return r; }
  Digest dg() { Digest d; for (int i = 0; i < 8; i++) d.v[i] = el(); return d; }
  uint32_t count(uint32_t max, const char* what) {
    uint32_t c = u32();
    if (c > max) throw std::runtime_error(std::string("proof: implausible count of ") + what);
    return c;
  }
  std::string str() {
    uint32_t len = count(1u << 16, "string bytes");
    if (n - pos < len) throw std::runtime_error("proof: truncated string");
    std::string s((const char*)b + pos, len);
    pos += len;
    return s;
  }
};

struct VPath { uint32_t leaf_idx = 0; std::vector<Digest> sib, inj; };
struct VLayer { uint32_t field = 0, row = 0; E6 p, q; VPath path; };
struct VRow { std::vector<uint32_t> b; std::vector<E6> e; };
struct VRows { VRow lo, hi; };
struct VSample { VRows top; VPath path; std::vector<VRows> inj; };
struct VGroupCV { std::vector<std::vector<E6>> b, e; };
struct VExposed { uint32_t idx, field; E6 v; };

struct VProof {
  std::string backend;
  std::map<std::string, std::vector<VExposed>> exposed;
  std::vector<Digest> commitments;
  std::vector<std::vector<VGroupCV>> cv;
  Digest levels_root;
  std::vector<std::vector<VLayer>> lq;   // extra levels x queries
  std::vector<Digest> fri_roots;
  uint32_t final_field = 0;
  std::vector<E6> final_poly;
  std::vector<std::vector<VLayer>> fq;   // queries x rounds r0..
  std::vector<std::vector<VSample>> ps;  // queries x committed trees
};

const uint32_t MAXC = 1u << 24;

VPath read_path(Reader& r) {
  VPath p;
  p.leaf_idx = r.u32();
  uint32_t ns = r.count(64, "siblings");
  for (uint32_t i = 0; i < ns; i++) p.sib.push_back(r.dg());
  uint32_t ni = r.count(MAXC, "injection leaves");
  for (uint32_t i = 0; i < ni; i++) p.inj.push_back(r.dg());
  return p;
}
VLayer read_layer(Reader& r) {
  VLayer l;
  l.field = r.u32();
  l.row = r.u32();
  l.p = r.e6();
  l.q = r.e6();
  l.path = read_path(r);
  return l;
}
VRow read_row(Reader& r) {
  VRow w;
  uint32_t nb = r.count(MAXC, "row base width");
  for (uint32_t i = 0; i < nb; i++) w.b.push_back(r.el());
  uint32_t ne = r.count(MAXC, "row ext width");
  for (uint32_t i = 0; i < ne; i++) w.e.push_back(r.e6());
  return w;
}

// Field order of proof.Proof (proof/proof.go:31-51) in the canonical encoding.
VProof decode(const uint8_t* b, size_t n) {
  Reader r{b, n};
  VProof pf;
  pf.backend = r.str();
  uint32_t ne = r.count(MAXC, "exposed values");
  for (uint32_t i = 0; i < ne; i++) {
    std::string name = r.str();
    if (pf.exposed.count(name)) throw std::runtime_error("proof: exposed value listed twice: " + name);
    uint32_t k = r.count(MAXC, "exposed entries");
    std::vector<VExposed> es;
    for (uint32_t j = 0; j < k; j++) {
      VExposed e;
      e.idx = r.u32();
      e.field = r.u32();
      e.v = r.e6();
      es.push_back(e);
    }
    pf.exposed[name] = es;
  }
  uint32_t nc = r.count(MAXC, "commitments");
  for (uint32_t i = 0; i < nc; i++) pf.commitments.push_back(r.dg());
  uint32_t nt = r.count(MAXC, "claimed-value batches");
  pf.cv.resize(nt);
  for (auto& t : pf.cv) {
    uint32_t ng = r.count(MAXC, "groups");
    t.resize(ng);
    for (auto& g : t) {
      for (int part = 0; part < 2; part++) {
        auto& polys = part == 0 ? g.b : g.e;
        uint32_t np = r.count(MAXC, "polynomials");
        polys.resize(np);
        for (auto& vals : polys) {
          uint32_t k = r.count(1024, "shifts");
          for (uint32_t j = 0; j < k; j++) vals.push_back(r.e6());
        }
      }
    }
  }
  pf.levels_root = r.dg();
  uint32_t nl = r.count(MAXC, "extra levels");
  pf.lq.resize(nl);
  for (auto& set : pf.lq) {
    uint32_t k = r.count(MAXC, "level queries");
    for (uint32_t j = 0; j < k; j++) set.push_back(read_layer(r));
  }
  uint32_t nr = r.count(64, "FRI roots");
  for (uint32_t i = 0; i < nr; i++) pf.fri_roots.push_back(r.dg());
  pf.final_field = r.u32();
  uint32_t nf = r.count(MAXC, "final polynomial");
  for (uint32_t i = 0; i < nf; i++) pf.final_poly.push_back(r.e6());
  uint32_t nq = r.count(MAXC, "FRI queries");
  pf.fq.resize(nq);
  for (auto& q : pf.fq) {
    uint32_t k = r.count(64, "FRI layers");
    for (uint32_t j = 0; j < k; j++) q.push_back(read_layer(r));
  }
  if (r.u32() != 0) throw std::runtime_error("proof: proofs of work present, grinding is off");
  uint32_t nps = r.count(MAXC, "point samplings");
  pf.ps.resize(nps);
  for (auto& q : pf.ps) {
    uint32_t k = r.count(MAXC, "sampled batches");
    q.resize(k);
    for (auto& s : q) {
      s.top.lo = read_row(r);
      s.top.hi = read_row(r);
      s.path = read_path(r);
      uint32_t ni = r.count(MAXC, "sampled injections");
      s.inj.resize(ni);
      for (auto& rows : s.inj) { rows.lo = read_row(r); rows.hi = read_row(r); }
    }
  }
  if (r.pos != n) throw std::runtime_error("proof: trailing bytes");
  return pf;
}

// ------------------------------------------------------------ helpers
int lg2(uint64_t x) { int k = 0; while ((1ull << k) < x) k++; return k; }

// leaf = Sponge(LEAF, 2nB, 2nE, lo.base, hi.base, lo.ext, hi.ext) (internal/fri/hash.go:39-57)
Digest pair_leaf(const VRows& r) {
  Sponge h;
  h.write((uint32_t)LEAF_TAG);
  h.write((uint32_t)(2 * r.lo.b.size()));
  h.write((uint32_t)(2 * r.lo.e.size()));
  for (uint32_t x : r.lo.b) h.write(x);
  for (uint32_t x : r.hi.b) h.write(x);
  for (auto& x : r.lo.e) h.write_e6(x);
  for (auto& x : r.hi.e) h.write_e6(x);
  return h.sum();
}
Digest layer_leaf(const VLayer& l) {
  VRows r;
  r.lo.e.push_back(l.p);
  r.hi.e.push_back(l.q);
  return pair_leaf(r);
}
Digest hnode(const Digest& l, const Digest& r) { return node_compress(NODE_TAG, l, r); }

// internal/merkle/tree.go:392-436: injections of each width fold in schedule
// order after the level of that width is reached.
bool verify_path(const Digest& root, const VPath& p, const Digest& leaf, const std::vector<size_t>& widths) {
  if (p.inj.size() != widths.size()) return false;
  size_t depth = p.sib.size(), prev = (size_t)1 << depth;
  for (size_t w : widths) {
    if (!w || (w & (w - 1)) || w > prev) return false;
    prev = w;
  }
  Digest h = leaf;
  uint64_t idx = p.leaf_idx;
  size_t next = 0;
  auto fold = [&](size_t width) {
    for (; next < widths.size() && widths[next] == width; next++) h = hnode(h, p.inj[next]);
  };
  fold((size_t)1 << depth);
  for (size_t k = 0; k < depth; k++) {
    h = (idx & 1) == 0 ? hnode(h, p.sib[k]) : hnode(p.sib[k], h);
    idx >>= 1;
    fold((size_t)1 << (depth - k - 1));
  }
  return next == widths.size() && digest_eq(h, root);
}

// L_i(zeta) = (zeta^n - 1)/n * w^i / (zeta - w^i)  (internal/poly/utils.go:66-104)
E6 lagrange_at(const E6& z, size_t n, size_t i) {
  uint32_t wi = pow(root_of_unity(n), i);
  E6 common = e6_mul_base(e6_sub(e6_pow(z, n), e6_one()), inv((uint32_t)(n % P)));
  return e6_mul(e6_mul_base(common, wi), e6_inv(e6_sub(z, e6_from_base(wi))));
}

[[noreturn]] void fail(const std::string& s) { throw std::runtime_error("verify: " + s); }

struct Verifier {
  const Program& pg;
  uint32_t nq;
  Prover lay;  // layout only (setup_layout), never a witness
  VProof pf;
  Transcript fs;
  std::vector<E6> coins, exposed;
  E6 zeta;
  std::map<std::pair<uint32_t, int>, E6> col_at;       // (column, normalized shift) -> value
  std::map<std::pair<uint32_t, uint32_t>, E6> chunk_at;  // (module, chunk) -> value
  std::vector<Digest> vk;     // setup roots (the verification key)
  std::vector<Digest> roots;  // per tree of the layout: setup roots, then the proof's commitments

  Verifier(const Program& p, uint32_t q) : pg(p), nq(q), lay(p, q) {}

  size_t mod_n(uint32_t m) const { return lay.mod_n(m); }

  std::string exposed_name(const PStep& st) const {
    return pg.columns[st.out].name + (st.type == STEP_LOGUP ? "_total" : "_end");
  }

  // ---------------------------------------------------------- transcript
  // verifier/verifier.go:167-252 (runtime init, deriveChallenges)
  void derive_challenges() {
    uint32_t R = pg.n_rounds;
    for (uint32_t r = 0; r < R; r++) fs.new_challenge(coin_name(r));
    fs.new_challenge("__zeta");
    std::string first = R > 0 ? coin_name(0) : "__zeta";
    fs.bind(first, string_to_elements(0x48415348, pf.backend));
    std::vector<uint32_t> sz = {0x53495a45, (uint32_t)lay.mod_order.size()};
    for (uint32_t m : lay.mod_order) sz.push_back((uint32_t)mod_n(m));
    fs.bind(first, sz);
    for (const Digest& d : vk) fs.bind(first, d.v, 8);  // setup roots (verifier/verifier.go:191-197)
    coins.assign(R, e6_zero());
    size_t ti = vk.size();
    for (uint32_t r = 0; r < R; r++) {
      if (ti < lay.trees.size() && !lay.trees[ti].air && lay.trees[ti].round == (int)r) {
        fs.bind(coin_name(r), roots[ti].v, 8);
        ti++;
      }
      for (const PStep& st : pg.steps) {  // BindExposedValues, board/logup.go:219-226
        if (st.round != r || (st.type != STEP_LOGUP && st.type != STEP_RATIO)) continue;
        for (const VExposed& e : pf.exposed.at(exposed_name(st))) {
          std::vector<uint32_t> w = {e.idx % P};
          for (int k = 0; k < 6; k++) w.push_back(e.v.c[k]);
          fs.bind(coin_name(r), w);
        }
      }
      coins[r] = digest_to_e6(fs.compute(coin_name(r)));
    }
    if (ti < lay.trees.size() && lay.trees[ti].air) {
      fs.bind("__zeta", roots[ti].v, 8);
      ti++;
    }
    if (ti != lay.trees.size()) fail("commitments out of layout order");
    zeta = digest_to_e6(fs.compute("__zeta"));
  }

  // ---------------------------------------------------------- shapes
  void check_shapes() {
    if (pf.backend != "poseidon2") fail("proof hash backend \"" + pf.backend + "\" is not poseidon2");
    const size_t n_setup = !lay.trees.empty() && lay.trees[0].setup ? 1 : 0;
    if (vk.size() != n_setup) fail("the verification key has " + std::to_string(vk.size()) + " setup roots, the layout " + std::to_string(n_setup));
    if (pf.commitments.size() + n_setup != lay.trees.size()) fail("commitment count differs from the layout");
    roots = vk;
    roots.insert(roots.end(), pf.commitments.begin(), pf.commitments.end());
    if (pf.cv.size() != lay.trees.size()) fail("claimed-value batches differ from the layout");
    for (size_t t = 0; t < lay.trees.size(); t++) {
      const auto& T = lay.trees[t];
      if (pf.cv[t].size() != T.groups.size()) fail("claimed-value groups differ from the layout");
      for (size_t g = 0; g < T.groups.size(); g++) {
        const auto& G = T.groups[g];
        const VGroupCV& cv = pf.cv[t][g];
        if (cv.b.size() != G.bcols.size() || cv.e.size() != G.ecols.size()) fail("claimed-value widths differ from the layout");
        for (size_t i = 0; i < G.bcols.size(); i++)
          if (cv.b[i].size() != lay.shifts_of(T, G.bcols[i]).size()) fail("claimed-value shift count differs");
        for (size_t i = 0; i < G.ecols.size(); i++)
          if (cv.e[i].size() != lay.shifts_of(T, G.ecols[i]).size()) fail("claimed-value shift count differs");
      }
    }
    // exposed values: one entry each (the totals and ends the steps expose)
    exposed.assign(0, e6_zero());
    for (const PStep& st : pg.steps) {
      if (st.type != STEP_LOGUP && st.type != STEP_RATIO) continue;
      auto it = pf.exposed.find(exposed_name(st));
      if (it == pf.exposed.end()) fail("exposed value " + exposed_name(st) + " missing");
      if (it->second.size() != 1) fail("exposed value " + exposed_name(st) + " must have exactly one entry");
      if (exposed.size() <= st.exposed) exposed.resize(st.exposed + 1);
      exposed[st.exposed] = it->second[0].field == 1 ? it->second[0].v : e6_from_base(it->second[0].v.c[0]);
    }
  }

  // ---------------------------------------------------------- values at zeta
  // loadClaimedValues (verifier/verifier.go:262-312)
  void load_claimed_values() {
    for (size_t t = 0; t < lay.trees.size(); t++) {
      const auto& T = lay.trees[t];
      for (size_t g = 0; g < T.groups.size(); g++) {
        const auto& G = T.groups[g];
        auto put = [&](uint32_t c, const std::vector<E6>& vals) {
          if (T.air) { chunk_at[{G.module, c}] = vals[0]; return; }
          std::vector<int> sh = lay.shifts_of(T, c);
          for (size_t k = 0; k < sh.size(); k++) col_at[{c, sh[k]}] = vals[k];
        };
        for (size_t i = 0; i < G.bcols.size(); i++) put(G.bcols[i], pf.cv[t][g].b[i]);
        for (size_t i = 0; i < G.ecols.size(); i++) put(G.ecols[i], pf.cv[t][g].e[i]);
      }
    }
  }

  // V(zeta) from claimed values, verifier columns (Lagrange, exposed values),
  // coins and constants (verifier/verifier.go:324-350, hookFns.go:34-97)
  E6 relation_at_zeta(uint32_t m) {
    std::vector<char> seen(lay.nodes.size(), 0);
    std::vector<uint32_t> order;
    lay.collect((uint32_t)lay.fold_root[m], seen, order);
    size_t n = mod_n(m);
    std::vector<E6> v(lay.nodes.size());
    for (uint32_t id : order) {
      const PNode& x = lay.nodes[id];
      switch (x.op) {
        case OP_COL: {
          const PColumn& col = pg.columns[x.a];
          int64_t sh = (int32_t)x.b;
          int s = (int)(((sh % (int64_t)n) + (int64_t)n) % (int64_t)n);
          if (col.kind == KIND_LAGRANGE) {
            int64_t row = col.param >= 0 ? col.param : (int64_t)n - 1 - (-(int64_t)col.param - 1);
            if (row < 0 || row >= (int64_t)n) fail("Lagrange column row out of range");
            v[id] = lagrange_at(zeta, n, (size_t)(((row - s) % (int64_t)n + (int64_t)n) % (int64_t)n));
          } else {
            auto it = col_at.find({x.a, s});
            if (it == col_at.end()) fail("no claimed value for column " + col.name);
            v[id] = it->second;
          }
          break;
        }
        case OP_COIN:
          if (x.a >= coins.size()) fail("coin of a round the program does not have");
          v[id] = coins[x.a];
          break;
        case OP_CONST: v[id] = e6_from_base(x.a % P); break;
        case OP_EXPAVG: v[id] = e6_mul_base(exposed.at(x.a), inv((uint32_t)(n % P))); break;
        case OP_EXPVAL: v[id] = exposed.at(x.a); break;
        case OP_ADD: v[id] = e6_add(v[x.a], v[x.b]); break;
        case OP_SUB: v[id] = e6_sub(v[x.a], v[x.b]); break;
        default: v[id] = e6_mul(v[x.a], v[x.b]); break;
      }
    }
    return v[lay.fold_root[m]];
  }

  // checkAIRRelations (verifier/verifier.go:394-432): V(zeta) = (zeta^N - 1) sum_i zeta^(iN) Q_i(zeta)
  void check_air() {
    for (uint32_t m : lay.mod_order) {
      if (lay.fold_root[m] < 0) continue;
      size_t n = mod_n(m);
      E6 zn = e6_pow(zeta, n), q = e6_zero(), zp = e6_one();
      for (uint32_t i = 0;; i++) {
        auto it = chunk_at.find({m, i});
        if (it == chunk_at.end()) break;
        q = e6_add(q, e6_mul(zp, it->second));
        zp = e6_mul(zp, zn);
      }
      E6 rhs = e6_mul(e6_sub(zn, e6_one()), q);
      if (!e6_eq(relation_at_zeta(m), rhs)) fail("AIR relation check failed for module " + pg.modules[m].name);
    }
  }

  // ---------------------------------------------------------- PCS
  struct Level { uint32_t module; size_t d; int intro; };
  std::vector<uint32_t> classes;  // modules with committed polynomials, sorted order
  std::vector<Level> levels;      // classes by size, descending (stable)
  std::vector<size_t> level_of;   // class index -> level
  E6 alpha;
  int r0 = 0;

  void pcs_verify() {
    for (uint32_t m : lay.mod_order) {
      bool has = false;
      for (auto& t : lay.trees) for (auto& g : t.groups) if (g.module == m) has = true;
      if (has) classes.push_back(m);
    }
    if (classes.empty()) fail("nothing committed");
    // alpha_DEEP over the claimed values in class -> batch -> group -> base -> ext -> shift
    // order (internal/fri/open.go:223-285)
    fs.new_challenge("alpha_DEEP");
    for (uint32_t m : classes)
      for (size_t t = 0; t < lay.trees.size(); t++)
        for (size_t g = 0; g < lay.trees[t].groups.size(); g++) {
          if (lay.trees[t].groups[g].module != m) continue;
          for (auto& vals : pf.cv[t][g].b) for (auto& v : vals) fs.bind("alpha_DEEP", v.c, 6);
          for (auto& vals : pf.cv[t][g].e) for (auto& v : vals) fs.bind("alpha_DEEP", v.c, 6);
        }
    alpha = digest_to_e6(fs.compute("alpha_DEEP"));

    std::vector<size_t> idx(classes.size());
    for (size_t i = 0; i < idx.size(); i++) idx[i] = i;
    std::stable_sort(idx.begin(), idx.end(), [&](size_t a, size_t b) { return mod_n(classes[a]) > mod_n(classes[b]); });
    level_of.assign(classes.size(), 0);
    for (size_t l = 0; l < idx.size(); l++) {
      size_t d = mod_n(classes[idx[l]]);
      levels.push_back({classes[idx[l]], d, lg2(((uint64_t)1 << MAX_LOG) / d)});
      level_of[idx[l]] = l;
    }
    std::vector<uint64_t> pos = fri_verify();
    check_point_samplings(pos);
    check_bridge(pos);
  }

  // fri.Verify + verifyExt + checkQueryExt (internal/fri/fri.go:751-1022,1430-1530);
  // returns the query positions s >> r0 << r0 (extractFRIQueryPositions).
  std::vector<uint64_t> fri_verify() {
    const int NR = MAX_LOG;
    size_t L = levels.size();
    r0 = levels[0].intro;
    if (r0 >= NR) fail("FRI: first level too small");
    if (pf.fri_roots.size() != (size_t)(NR - 1 - r0)) fail("FRI: wrong number of layer roots");
    if (pf.fq.size() != nq) fail("FRI: wrong number of queries");
    for (auto& q : pf.fq) if (q.size() != (size_t)(NR - r0)) fail("FRI: wrong number of query layers");
    if (pf.lq.size() != L - 1) fail("FRI: wrong number of level query sets");
    for (auto& s : pf.lq) if (s.size() != nq) fail("FRI: wrong number of level queries");
    if (pf.final_field != 1 || pf.final_poly.empty()) fail("FRI: final polynomial must be a non-empty extension vector");
    for (size_t l = 1; l < L; l++) fs.new_challenge("fri_level_" + std::to_string(l) + "_gamma");
    for (int j = 0; j < NR; j++) fs.new_challenge("fri_fold_" + std::to_string(j));
    for (uint32_t k = 0; k < nq; k++) fs.new_challenge("fri_query_" + std::to_string(k));
    std::vector<E6> gam(L);
    for (size_t l = 1; l < L; l++) {  // deriveLevelGammas (internal/fri/fri.go:443-459)
      std::string nm = "fri_level_" + std::to_string(l) + "_gamma";
      if (l == 1) fs.bind(nm, pf.levels_root.v, 8);
      gam[l] = digest_to_e6(fs.compute(nm));
    }
    Digest zero;
    memset(zero.v, 0, sizeof zero.v);
    for (int j = 0; j < r0; j++) {  // deriveEmptyRoundChallenges (internal/fri/fri.go:1039-1051)
      fs.bind("fri_fold_" + std::to_string(j), zero.v, 8);
      fs.compute("fri_fold_" + std::to_string(j));
    }
    std::vector<Digest> roots(NR);
    std::vector<E6> alphas(NR);
    for (int j = r0; j < NR; j++) {
      roots[j] = j == r0 ? pf.levels_root : pf.fri_roots[j - r0 - 1];
      std::string nm = "fri_fold_" + std::to_string(j);
      fs.bind(nm, roots[j].v, 8);
      alphas[j] = digest_to_e6(fs.compute(nm));
    }
    {
      std::vector<uint32_t> fin = {0x45585450, (uint32_t)pf.final_poly.size()};
      for (auto& v : pf.final_poly) for (int i = 0; i < 6; i++) fin.push_back(v.c[i]);
      fs.bind("fri_query_0", fin);
    }
    // levels-tree injection widths: pair leaves of every extra level
    std::vector<size_t> widths;
    for (size_t l = 1; l < L; l++) widths.push_back(RATE * levels[l].d / 2);
    std::map<int, std::vector<size_t>> at_round;
    for (size_t l = 1; l < L; l++) at_round[levels[l].intro].push_back(l);
    uint32_t inv2 = inv(2);
    std::vector<uint64_t> pos(nq);
    for (uint32_t k = 0; k < nq; k++) {
      Digest c = fs.compute("fri_query_" + std::to_string(k));
      uint64_t s = (((uint64_t)c.v[0] << 31) ^ (uint64_t)c.v[1]) % N_FRI;  // queryIndex
      if (k + 1 < nq) fs.bind("fri_query_" + std::to_string(k + 1), c.v, 8);
      const auto& fq = pf.fq[k];
      for (int j = r0; j < NR; j++) {
        const VLayer& layer = fq[j - r0];
        uint64_t row = s >> j, lo = row & ~(uint64_t)1;
        size_t nj = (size_t)(N_FRI >> j);
        if (layer.field != 1) fail("FRI: query layer is not an extension layer");
        if (layer.row != row) fail("FRI: query row differs from the transcript's");
        if (layer.path.leaf_idx != lo / 2) fail("FRI: path opens the wrong pair");
        if (j == r0) {  // verifyLevelsPath (internal/fri/fri.go:856-882)
          VPath path = layer.path;
          path.inj.clear();
          for (size_t l = 1; l < L; l++) {
            const VLayer& ld = pf.lq[l - 1][k];
            if (ld.field != 1) fail("FRI: level query is not an extension layer");
            // the levels tree authenticates it; a path of its own is not part of the encoding
            if (ld.path.leaf_idx || !ld.path.sib.empty() || !ld.path.inj.empty()) fail("FRI: level query carries a path");
            if (ld.row != (s >> levels[l].intro)) fail("FRI: level query row differs from the transcript's");
            path.inj.push_back(layer_leaf(ld));
          }
          if (!verify_path(roots[j], path, layer_leaf(layer), widths)) fail("FRI: levels tree path invalid");
        } else if (!layer.path.inj.empty() || !verify_path(roots[j], layer.path, layer_leaf(layer), {})) {
          fail("FRI: layer " + std::to_string(j) + " Merkle path invalid");
        }
        E6 p = layer.p, q = layer.q;
        if (j == r0)
          for (size_t l : at_round[r0]) {
            const VLayer& ld = pf.lq[l - 1][k];
            p = e6_add(p, e6_mul(ld.p, gam[l]));
            q = e6_add(q, e6_mul(ld.q, gam[l]));
          }
        // x^-1 = w_nj^-bitrev(i, nj/2) for pair i (internal/fri/fri.go:1113-1118)
        uint32_t xinv = pow(inv(root_of_unity(nj)), bitrev((uint32_t)(lo >> 1), lg2(nj / 2)));
        E6 expected = e6_add(e6_mul_base(e6_add(p, q), inv2),
                             e6_mul(e6_mul_base(e6_mul_base(e6_sub(p, q), inv2), xinv), alphas[j]));
        if (j < NR - 1) {
          uint64_t nrow = row >> 1;
          const VLayer& next = fq[j + 1 - r0];
          bool leaf_p = (nrow & 1) == 0;
          auto it = at_round.find(j + 1);
          if (it != at_round.end())
            for (size_t l : it->second) {
              const VLayer& ld = pf.lq[l - 1][k];
              if (ld.row != nrow) fail("FRI: level query row differs at its intro round");
              expected = e6_add(expected, e6_mul(leaf_p ? ld.p : ld.q, gam[l]));
            }
          if (!e6_eq(expected, leaf_p ? next.p : next.q)) fail("FRI: fold mismatch at round " + std::to_string(j + 1));
        } else {
          uint64_t f = s >> NR;
          if (f >= pf.final_poly.size() || !e6_eq(expected, pf.final_poly[f])) fail("FRI: folded value does not match the final polynomial");
        }
      }
      pos[k] = (uint64_t)fq[0].row << r0;
    }
    return pos;
  }

  // groups of a tree in decreasing row count, ties in declaration order
  std::vector<size_t> injection_order(size_t t) const {
    const auto& G = lay.trees[t].groups;
    std::vector<size_t> o(G.size());
    for (size_t i = 0; i < o.size(); i++) o[i] = i;
    std::stable_sort(o.begin(), o.end(), [&](size_t a, size_t b) { return mod_n(G[a].module) > mod_n(G[b].module); });
    return o;
  }
  static bool row_width(const VRow& r, const Prover::Group& g) { return r.b.size() == g.bcols.size() && r.e.size() == g.ecols.size(); }

  // verifyAllPointSamplings / verifyOneWMerkleProof (internal/fri/verify.go:277-455)
  void check_point_samplings(const std::vector<uint64_t>& pos) {
    if (pf.ps.size() != nq) fail("point samplings: wrong number of queries");
    const int LOGN = lg2(N_FRI);
    for (uint32_t k = 0; k < nq; k++) {
      if (pf.ps[k].size() != lay.trees.size()) fail("point samplings: wrong number of batches");
      for (size_t t = 0; t < lay.trees.size(); t++) {
        const VSample& sp = pf.ps[k][t];
        const auto& G = lay.trees[t].groups;
        std::vector<size_t> ord = injection_order(t);
        if (sp.inj.size() != ord.size() - 1) fail("point samplings: wrong number of injected groups");
        size_t top_rows = RATE * mod_n(G[ord[0]].module), top_pairs = top_rows / 2;
        if (!row_width(sp.top.lo, G[ord[0]]) || !row_width(sp.top.hi, G[ord[0]])) fail("point samplings: top row width");
        std::vector<size_t> widths;
        for (size_t i = 1; i < ord.size(); i++) {
          if (!row_width(sp.inj[i - 1].lo, G[ord[i]]) || !row_width(sp.inj[i - 1].hi, G[ord[i]])) fail("point samplings: injected row width");
          widths.push_back(RATE * mod_n(G[ord[i]].module) / 2);
        }
        if (!sp.path.inj.empty() && sp.path.inj.size() != widths.size()) fail("point samplings: injection leaves count");
        uint64_t trow = pos[k] >> (LOGN - lg2(top_rows)), tlo = trow & ~(uint64_t)1;
        if (sp.path.leaf_idx != tlo / 2) fail("point samplings: path opens the wrong pair");
        size_t depth = (size_t)lg2(top_pairs);
        if (sp.path.sib.size() != depth) fail("point samplings: path depth");
        Digest h = pair_leaf(sp.top);
        uint64_t idx = sp.path.leaf_idx;
        size_t next = 0;
        auto fold = [&](size_t width) {
          for (; next < widths.size() && widths[next] == width; next++) {
            size_t rows = 2 * widths[next];
            uint64_t row = pos[k] >> (LOGN - lg2(rows)), lo = row & ~(uint64_t)1;
            if (idx != lo / 2) fail("point samplings: injected pair off the path");
            Digest d = pair_leaf(sp.inj[next]);
            if (!sp.path.inj.empty() && !digest_eq(d, sp.path.inj[next])) fail("point samplings: injection pair hash mismatch");
            h = hnode(h, d);
          }
        };
        fold(top_pairs);
        for (size_t s = 0; s < depth; s++) {
          h = (idx & 1) == 0 ? hnode(h, sp.path.sib[s]) : hnode(sp.path.sib[s], h);
          idx >>= 1;
          fold((size_t)1 << (depth - s - 1));
        }
        if (next != widths.size() || !digest_eq(h, roots[t]))
          fail("point samplings: Merkle path does not authenticate under batch " + std::to_string(t) + "'s root");
      }
    }
  }

  // checkFRIBridgeByPolynomial (internal/fri/verify.go:499-700): DQ_c(X), DQ_c(-X)
  // recomputed from the opened rows and the claimed values equal the FRI level leaves.
  void check_bridge(const std::vector<uint64_t>& pos) {
    const int LOGN = lg2(N_FRI);
    for (uint32_t k = 0; k < nq; k++) {
      for (size_t ci = 0; ci < classes.size(); ci++) {
        uint32_t m = classes[ci];
        size_t n = mod_n(m), rat = RATE * n;
        uint64_t row = pos[k] >> (LOGN - lg2(rat)), lo = row & ~(uint64_t)1, hi = lo + 1;
        uint32_t g = root_of_unity(rat);
        uint32_t X = pow(g, bitrev((uint32_t)lo, lg2(rat))), Xh = pow(g, bitrev((uint32_t)hi, lg2(rat)));
        if (Xh != neg(X)) fail("bridge: companion row is not -X");
        E6 x = e6_from_base(X), nx = e6_from_base(neg(X));
        uint32_t w = root_of_unity(n);
        E6 dp = e6_zero(), dq = e6_zero(), run = e6_one();
        for (size_t t = 0; t < lay.trees.size(); t++) {
          const auto& T = lay.trees[t];
          std::vector<size_t> ord = injection_order(t);
          for (size_t gi = 0; gi < T.groups.size(); gi++) {
            const auto& G = T.groups[gi];
            if (G.module != m) continue;
            size_t at = (size_t)(std::find(ord.begin(), ord.end(), gi) - ord.begin());
            const VRows& raw = at == 0 ? pf.ps[k][t].top : pf.ps[k][t].inj[at - 1];
            auto bundle = [&](const std::vector<int>& shifts, const std::vector<E6>& vals, const E6& lp, const E6& lq) {
              E6 bp = e6_zero(), bq = e6_zero();
              for (size_t s = 0; s < shifts.size(); s++) {
                E6 zs = e6_mul_base(zeta, pow(w, (uint64_t)shifts[s]));
                bp = e6_add(bp, e6_mul(e6_sub(vals[s], lp), e6_inv(e6_sub(zs, x))));
                bq = e6_add(bq, e6_mul(e6_sub(vals[s], lq), e6_inv(e6_sub(zs, nx))));
              }
              dp = e6_add(dp, e6_mul(bp, run));
              dq = e6_add(dq, e6_mul(bq, run));
              run = e6_mul(run, alpha);
            };
            for (size_t i = 0; i < G.bcols.size(); i++)
              bundle(lay.shifts_of(T, G.bcols[i]), pf.cv[t][gi].b[i], e6_from_base(raw.lo.b[i]), e6_from_base(raw.hi.b[i]));
            for (size_t i = 0; i < G.ecols.size(); i++)
              bundle(lay.shifts_of(T, G.ecols[i]), pf.cv[t][gi].e[i], raw.lo.e[i], raw.hi.e[i]);
          }
        }
        size_t l = level_of[ci];
        const VLayer& want = l == 0 ? pf.fq[k][0] : pf.lq[l - 1][k];
        if (!e6_eq(dp, want.p) || !e6_eq(dq, want.q))
          fail("bridge: DEEP quotient of module " + pg.modules[m].name + " differs from its FRI level at query " + std::to_string(k));
      }
    }
  }

  // checkProductBus / checkLogupBus (verifier/verifier.go:352-392): the
  // running-ratio ends of a product bus multiply to one, the logup totals of
  // a logup bus sum to zero.  `buses` lists them as "P:name,name;L:name,...".
  void check_buses(const std::string& buses) {
    size_t i = 0;
    while (i < buses.size()) {
      size_t j = buses.find(';', i);
      if (j == std::string::npos) j = buses.size();
      std::string bus = buses.substr(i, j - i);
      i = j + 1;
      if (bus.empty()) continue;
      if (bus.size() < 2 || (bus[0] != 'P' && bus[0] != 'L') || bus[1] != ':') fail("bad bus list");
      bool product = bus[0] == 'P';
      E6 acc = product ? e6_one() : e6_zero();
      size_t a = 2;
      while (a <= bus.size()) {
        size_t b = bus.find(',', a);
        if (b == std::string::npos) b = bus.size();
        std::string name = bus.substr(a, b - a);
        a = b + 1;
        auto it = pf.exposed.find(name);
        if (it == pf.exposed.end() || it->second.size() != 1) fail("bus value " + name + " must be exposed with exactly one entry");
        const VExposed& e = it->second[0];
        E6 v = e.field == 1 ? e.v : e6_from_base(e.v.c[0]);
        acc = product ? e6_mul(acc, v) : e6_add(acc, v);
      }
      if (product && !e6_eq(acc, e6_one())) fail("the running ratios of a product bus do not multiply to one");
      if (!product && !e6_is_zero(acc)) fail("the logup totals of a bus do not sum to zero");
    }
  }

  // Verify (verifier/verifier.go:487-533)
  void verify(const uint8_t* b, size_t n, const std::string& buses) {
    pf = decode(b, n);
    lay.setup_layout();
    check_shapes();
    derive_challenges();
    load_claimed_values();
    check_buses(buses);
    check_air();
    pcs_verify();
  }
};

}  // namespace

void oracle_verify_bytes(const Program& pg, const uint8_t* proof, size_t len, uint32_t num_queries, const std::string& buses,
                         const std::vector<Digest>& setup_roots) {
  Verifier v(pg, num_queries);
  v.vk = setup_roots;
  v.verify(proof, len, buses);
}

}  // namespace orc
