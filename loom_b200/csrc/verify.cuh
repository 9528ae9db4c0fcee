// Verifier of the canonical proof encoding for the Poseidon2 backend
// (verifier/verifier.go:119-533, internal/fri/verify.go, internal/fri/fri.go:751-1022,
// internal/merkle/tree.go:392-436), with the bulk of the work on the GPU:
//  * the host decodes the proof, replays the transcript, checks the buses,
//    the AIR relation at zeta and the FRI fold chain of every query;
//  * k_verify_paths recomputes every Merkle opening (the opened row pairs of
//    each batch hashed into leaves, injected groups folded in at their
//    widths, the path walked to the root; the levels tree and the FRI layer
//    trees take the same form), one job per thread;
//  * k_verify_bridge recomputes, for every query and DEEP class, DQ(X) and
//    DQ(-X) from the opened rows and the claimed values and compares them
//    with the FRI level values.
// Field words are Montgomery on the device and on the host; the proof's
// canonical words are converted on decoding.
#pragma once
#include "prover.cuh"

namespace lg {

// ---------------------------------------------------------------- device side
// One Merkle opening: groups in injection order (the first is the leaf level,
// its pair index leaf_idx); group g's lo and hi rows (nb + 6 ne words each)
// follow one another in `words` from rows_off; shape[g] = (nb, ne, log2 of
// its pair width).  Injected pair digests given by the proof (inj_off, or
// ~0) must equal the recomputed ones.
constexpr uint32_t VJ_MAX_GROUPS = 64;
struct VerifyJob {
  uint64_t rows_off, sib_off, inj_off, root_off;
  uint32_t shape_off, n_groups, leaf_idx, depth;
};
struct VSponge {
  uint32_t s[24], blk[16];
  int len = 0;
  __device__ VSponge() {
    for (int i = 0; i < 24; i++) s[i] = 0;
    for (int i = 0; i < 16; i++) blk[i] = 0;
  }
  __device__ void write(uint32_t x) {
    blk[len++] = x;
    if (len == 16) {
      for (int i = 0; i < 16; i++) s[i] = blk[i];
      p2_permute(s);
      len = 0;
    }
  }
  __device__ void sum(uint32_t out[8]) {
    if (len > 0) {
      for (int i = 0; i < len; i++) s[i] = blk[i];
      p2_permute(s);
      len = 0;
    }
    for (int i = 0; i < 8; i++) out[i] = s[i];
  }
};
// leaf = Sponge(LEAF, 2nb, 2ne, lo.base, hi.base, lo.ext, hi.ext) (internal/fri/hash.go:39-57)
__device__ void v_pair_leaf(const uint32_t* lo, const uint32_t* hi, uint32_t nb, uint32_t ne, uint32_t out[8]) {
  VSponge h;
  h.write(to_mont(LEAF_TAG));
  h.write(to_mont(2 * nb));
  h.write(to_mont(2 * ne));
  for (uint32_t i = 0; i < nb; i++) h.write(lo[i]);
  for (uint32_t i = 0; i < nb; i++) h.write(hi[i]);
  for (uint32_t i = 0; i < 6 * ne; i++) h.write(lo[nb + i]);
  for (uint32_t i = 0; i < 6 * ne; i++) h.write(hi[nb + i]);
  h.sum(out);
}
// bad[j] = 0 when job j authenticates, else 1 (path) or 2 (injection leaf mismatch)
__global__ void k_verify_paths(const VerifyJob* jobs, uint32_t n_jobs, const uint32_t* words, const uint32_t* shapes,
                               uint32_t* bad) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n_jobs) return;
  const VerifyJob J = jobs[j];
  const uint32_t* sh = shapes + J.shape_off;
  const uint32_t* row = words + J.rows_off;
  uint32_t h[8], d[8];
  uint32_t status = 0;
  {
    const uint32_t w0 = sh[0] + 6 * sh[1];
    v_pair_leaf(row, row + w0, sh[0], sh[1], h);
    row += 2 * w0;
  }
  uint32_t next = 1, idx = J.leaf_idx;
  const uint32_t tag = to_mont(NODE_TAG);
  auto fold = [&](uint32_t logw) {
    for (; next < J.n_groups && sh[3 * next + 2] == logw; next++) {
      const uint32_t nb = sh[3 * next], ne = sh[3 * next + 1], w = nb + 6 * ne;
      v_pair_leaf(row, row + w, nb, ne, d);
      row += 2 * w;
      if (J.inj_off != ~0ull)
        for (int k = 0; k < 8; k++)
          if (words[J.inj_off + 8 * (uint64_t)(next - 1) + k] != d[k]) status = 2;
      p2_compress(tag, h, d, h);
    }
  };
  fold(J.depth);
  for (uint32_t k = 0; k < J.depth; k++) {
    const uint32_t* sib = words + J.sib_off + 8 * (uint64_t)k;
    uint32_t s[8];
    for (int q = 0; q < 8; q++) s[q] = sib[q];
    if ((idx & 1) == 0) p2_compress(tag, h, s, h);
    else p2_compress(tag, s, h, h);
    idx >>= 1;
    fold(J.depth - k - 1);
  }
  if (next != J.n_groups) status = 1;
  for (int q = 0; q < 8; q++)
    if (h[q] != words[J.root_off + q]) status = 1;
  bad[j] = status;
}

// DEEP bridge (internal/fri/verify.go:499-700): per (query, class) job, terms
// [t0, t1) of one polynomial and shift each: sum over terms of
// scale (v - P(x)) / (z_s - x) at x = X and x = -X, compared with the level
// values want_p, want_q.
struct BridgeTerm { uint64_t lo_off, hi_off; uint32_t ext, cv, zs, scale; };
struct BridgeJob { uint32_t t0, t1, x; E6 want_p, want_q; };
__global__ void k_verify_bridge(const BridgeJob* jobs, uint32_t n_jobs, const BridgeTerm* terms, const uint32_t* words,
                                const E6* cvs, const E6* zs, const E6* scales, uint32_t* bad) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n_jobs) return;
  const BridgeJob J = jobs[j];
  const E6 X = e6_base(J.x), NX = e6_base(neg(J.x));
  E6 dp = e6_zero(), dq = e6_zero();
  for (uint32_t t = J.t0; t < J.t1; t++) {
    const BridgeTerm T = terms[t];
    E6 lp, lq;
    if (T.ext) {
      for (int k = 0; k < 6; k++) { lp.c[k] = words[T.lo_off + k]; lq.c[k] = words[T.hi_off + k]; }
    } else {
      lp = e6_base(words[T.lo_off]);
      lq = e6_base(words[T.hi_off]);
    }
    const E6 v = cvs[T.cv], z = zs[T.zs], sc = scales[T.scale];
    dp = e6_add(dp, e6_mul(sc, e6_mul(e6_sub(v, lp), e6_inv(e6_sub(z, X)))));
    dq = e6_add(dq, e6_mul(sc, e6_mul(e6_sub(v, lq), e6_inv(e6_sub(z, NX)))));
  }
  bad[j] = (e6_eq(dp, J.want_p) && e6_eq(dq, J.want_q)) ? 0u : 1u;
}

// ---------------------------------------------------------------- host side
struct ProofVerifier {
  Ctx& c;
  Prover lay;  // the program's layout (setup_layout), never a witness
  uint32_t nq;
  // decoded proof (Montgomery)
  struct VPath { uint32_t leaf_idx = 0; std::vector<Digest> sib, inj; };
  struct VLayer { uint32_t field = 0, row = 0; E6 p, q; VPath path; };
  struct VRow { std::vector<uint32_t> w; uint32_t nb = 0, ne = 0; };  // nb base words then 6 per ext value
  struct VSample { VRow top_lo, top_hi; VPath path; std::vector<std::pair<VRow, VRow>> inj; };
  struct VExposed { uint32_t idx, field; E6 v; };
  std::string backend;
  std::map<std::string, std::vector<VExposed>> exposed_by_name;
  std::vector<Digest> commitments, roots;
  std::vector<std::vector<std::vector<std::vector<E6>>>> cv;  // tree, group, poly (base then ext), shift
  Digest levels_root{};
  std::vector<std::vector<VLayer>> lq, fq;
  std::vector<Digest> fri_roots;
  uint32_t final_field = 0;
  std::vector<E6> final_poly;
  std::vector<std::vector<VSample>> ps;
  // derived
  std::vector<E6> coins, exposed;
  E6 zeta{}, alpha{};
  std::map<std::pair<uint32_t, int>, E6> col_at;
  std::map<std::pair<uint32_t, uint32_t>, E6> chunk_at;

  ProofVerifier(Ctx& ctx, const uint32_t* words, size_t nwords, uint32_t q) : c(ctx), lay(ctx, words, nwords, q), nq(q) {}

  [[noreturn]] static void reject(const std::string& why) { throw Error(LG_ERR_INVALID, "proof rejected: " + why); }

  // ------------------------------------------------------------ decoding
  struct Reader {
    const uint8_t* b;
    size_t n, pos = 0;
    uint32_t u32() {
      if (n - pos < 4) reject("truncated");
      uint32_t x = ((uint32_t)b[pos] << 24) | ((uint32_t)b[pos + 1] << 16) | ((uint32_t)b[pos + 2] << 8) | (uint32_t)b[pos + 3];
      pos += 4;
      return x;
    }
    uint32_t el() {
      uint32_t x = u32();
      if (x >= P) reject("field element not reduced");
      return to_mont(x);
    }
    E6 e6() { E6 r; for (int i = 0; i < 6; i++) r.c[i] = el(); return r; }
    Digest dg() { Digest d; for (int i = 0; i < 8; i++) d.v[i] = el(); return d; }
    uint32_t count(uint32_t max) {
      uint32_t c = u32();
      if (c > max) reject("implausible count");
      return c;
    }
    std::string str() {
      uint32_t len = count(1u << 16);
      if (n - pos < len) reject("truncated string");
      std::string s((const char*)b + pos, len);
      pos += len;
      return s;
    }
    VPath path() {
      VPath p;
      p.leaf_idx = u32();
      uint32_t ns = count(64);
      for (uint32_t i = 0; i < ns; i++) p.sib.push_back(dg());
      uint32_t ni = count(1u << 24);
      for (uint32_t i = 0; i < ni; i++) p.inj.push_back(dg());
      return p;
    }
    VLayer layer() {
      VLayer l;
      l.field = u32();
      l.row = u32();
      l.p = e6();
      l.q = e6();
      l.path = path();
      return l;
    }
    VRow row() {
      VRow r;
      r.nb = count(1u << 24);
      for (uint32_t i = 0; i < r.nb; i++) r.w.push_back(el());
      r.ne = count(1u << 24);
      for (uint32_t i = 0; i < r.ne; i++) { E6 e = e6(); r.w.insert(r.w.end(), e.c, e.c + 6); }
      return r;
    }
  };
  void decode(const uint8_t* b, size_t n) {
    Reader r{b, n};
    backend = r.str();
    const uint32_t ne = r.count(1u << 24);
    for (uint32_t i = 0; i < ne; i++) {
      std::string name = r.str();
      if (exposed_by_name.count(name)) reject("exposed value listed twice");
      uint32_t k = r.count(1u << 24);
      std::vector<VExposed> es;
      for (uint32_t j = 0; j < k; j++) {
        VExposed e;
        e.idx = r.u32();
        e.field = r.u32();
        e.v = r.e6();
        es.push_back(e);
      }
      exposed_by_name[name] = es;
    }
    const uint32_t nc = r.count(1u << 24);
    for (uint32_t i = 0; i < nc; i++) commitments.push_back(r.dg());
    cv.resize(r.count(1u << 24));
    for (auto& t : cv) {
      t.resize(r.count(1u << 24));
      for (auto& g : t) {
        for (int part = 0; part < 2; part++) {
          const uint32_t np = r.count(1u << 24);
          for (uint32_t p = 0; p < np; p++) {
            std::vector<E6> vals;
            const uint32_t k = r.count(1024);
            for (uint32_t s = 0; s < k; s++) vals.push_back(r.e6());
            g.push_back(vals);
          }
          if (part == 0) g.push_back({});  // separator between base and ext polynomials
        }
      }
    }
    levels_root = r.dg();
    lq.resize(r.count(1u << 24));
    for (auto& set : lq) {
      const uint32_t k = r.count(1u << 24);
      for (uint32_t j = 0; j < k; j++) set.push_back(r.layer());
    }
    const uint32_t nr = r.count(64);
    for (uint32_t i = 0; i < nr; i++) fri_roots.push_back(r.dg());
    final_field = r.u32();
    const uint32_t nf = r.count(1u << 24);
    for (uint32_t i = 0; i < nf; i++) final_poly.push_back(r.e6());
    fq.resize(r.count(1u << 24));
    for (auto& q : fq) {
      const uint32_t k = r.count(64);
      for (uint32_t j = 0; j < k; j++) q.push_back(r.layer());
    }
    if (r.u32() != 0) reject("proofs of work present, grinding is off");
    ps.resize(r.count(1u << 24));
    for (auto& q : ps) {
      q.resize(r.count(1u << 24));
      for (auto& s : q) {
        s.top_lo = r.row();
        s.top_hi = r.row();
        s.path = r.path();
        s.inj.resize(r.count(1u << 24));
        for (auto& x : s.inj) { x.first = r.row(); x.second = r.row(); }
      }
    }
    if (r.pos != n) reject("trailing bytes");
  }

  std::vector<int> shifts_of(size_t t, uint32_t col) const {
    if (lay.trees[t].air) return {0};
    auto it = lay.col_shifts.find(col);
    return it == lay.col_shifts.end() ? std::vector<int>{} : it->second;
  }
  std::string exposed_name(const Step& st) const {
    return lay.pg.columns[st.out].name + (st.type == STEP_LOGUP ? "_total" : "_end");
  }
  size_t mod_n(uint32_t m) const { return lay.mod_n(m); }

  // ------------------------------------------------------------ shapes
  void check_shapes(const Digest* setup_root) {
    if (backend != "poseidon2") reject("hash backend \"" + backend + "\" is not poseidon2");
    const auto& T = lay.trees;
    const size_t n_setup = !T.empty() && T[0].setup ? 1 : 0;
    if ((setup_root != nullptr) != (n_setup == 1)) reject("the verification key does not match the program's setup");
    if (commitments.size() + n_setup != T.size()) reject("commitment count differs from the layout");
    if (n_setup) roots.push_back(*setup_root);
    roots.insert(roots.end(), commitments.begin(), commitments.end());
    if (cv.size() != T.size()) reject("claimed-value batches differ from the layout");
    for (size_t t = 0; t < T.size(); t++) {
      if (cv[t].size() != T[t].groups.size()) reject("claimed-value groups differ from the layout");
      for (size_t g = 0; g < T[t].groups.size(); g++) {
        const auto& G = T[t].groups[g];
        const auto& V = cv[t][g];
        if (V.size() != G.bcols.size() + 1 + G.ecols.size()) reject("claimed-value widths differ from the layout");
        for (size_t i = 0; i < G.bcols.size(); i++)
          if (V[i].size() != shifts_of(t, G.bcols[i]).size()) reject("claimed-value shift count differs");
        for (size_t i = 0; i < G.ecols.size(); i++)
          if (V[G.bcols.size() + 1 + i].size() != shifts_of(t, G.ecols[i]).size()) reject("claimed-value shift count differs");
      }
    }
    exposed.assign(lay.n_exposed(), e6_zero());
    for (const Step& st : lay.pg.steps) {
      if (!exposes(st.type)) continue;
      auto it = exposed_by_name.find(exposed_name(st));
      if (it == exposed_by_name.end() || it->second.size() != 1) reject("exposed value " + exposed_name(st) + " missing");
      exposed[st.exposed] = it->second[0].field == 1 ? it->second[0].v : e6_base(it->second[0].v.c[0]);
    }
  }
  // cv[t][g] holds the base polynomials' values, an empty separator, then the
  // extension polynomials'
  size_t ext_index(size_t t, size_t g, size_t i) const { return lay.trees[t].groups[g].bcols.size() + 1 + i; }

  // ------------------------------------------------------------ transcript
  void derive_challenges() {
    Transcript& fs = lay.fs;
    const uint32_t R = lay.pg.n_rounds;
    for (uint32_t r = 0; r < R; r++) fs.add(coin_name(r));
    fs.add("__zeta");
    const std::string first = coin_name(0);
    auto hb = string_to_elements(0x48415348u, backend);
    fs.bind(first, hb.data(), hb.size());
    std::vector<uint32_t> sz = {to_mont(0x53495a45u), to_mont((uint32_t)lay.mod_order.size())};
    for (uint32_t m : lay.mod_order) sz.push_back(to_mont((uint32_t)mod_n(m)));
    fs.bind(first, sz.data(), sz.size());
    size_t ti = 0;
    if (!lay.trees.empty() && lay.trees[0].setup) {
      fs.bind(first, roots[0].v, 8);
      ti = 1;
    }
    coins.assign(R, e6_zero());
    for (uint32_t r = 0; r < R; r++) {
      if (ti < lay.trees.size() && !lay.trees[ti].air && lay.trees[ti].round == (int)r) {
        fs.bind(coin_name(r), roots[ti].v, 8);
        ti++;
      }
      for (const Step& st : lay.pg.steps) {
        if (st.round != r || !exposes(st.type)) continue;
        uint32_t w[7] = {0};
        for (int k = 0; k < 6; k++) w[1 + k] = exposed[st.exposed].c[k];
        fs.bind(coin_name(r), w, 7);
      }
      coins[r] = digest_e6(fs.compute(coin_name(r)));
    }
    if (ti < lay.trees.size() && lay.trees[ti].air) {
      fs.bind("__zeta", roots[ti].v, 8);
      ti++;
    }
    if (ti != lay.trees.size()) reject("commitments out of layout order");
    zeta = digest_e6(fs.compute("__zeta"));
  }

  // ------------------------------------------------------------ buses and AIR
  void check_buses(const char* buses) {
    std::string spec = buses ? buses : "";
    size_t i = 0;
    while (i < spec.size()) {
      size_t j = spec.find(';', i);
      if (j == std::string::npos) j = spec.size();
      std::string bus = spec.substr(i, j - i);
      i = j + 1;
      if (bus.empty()) continue;
      if (bus.size() < 2 || (bus[0] != 'P' && bus[0] != 'L') || bus[1] != ':') throw Error(LG_ERR_INVALID, "bad bus list");
      const bool product = bus[0] == 'P';
      E6 acc = product ? e6_one() : e6_zero();
      size_t a = 2;
      while (a <= bus.size()) {
        size_t b = bus.find(',', a);
        if (b == std::string::npos) b = bus.size();
        const std::string name = bus.substr(a, b - a);
        a = b + 1;
        auto it = exposed_by_name.find(name);
        if (it == exposed_by_name.end() || it->second.size() != 1) reject("bus value " + name + " not exposed");
        const VExposed& e = it->second[0];
        const E6 v = e.field == 1 ? e.v : e6_base(e.v.c[0]);
        acc = product ? e6_mul(acc, v) : e6_add(acc, v);
      }
      if (product && !e6_eq(acc, e6_one())) reject("the running ratios of a product bus do not multiply to one");
      if (!product && !e6_eq(acc, e6_zero())) reject("the logup totals of a bus do not sum to zero");
    }
  }
  // L_i(zeta) = (zeta^n - 1)/n w^i / (zeta - w^i)  (internal/poly/utils.go:66-104)
  E6 lagrange_at(size_t n, size_t i) const {
    const uint32_t wi = mont_pow(root_of_unity_mont(__builtin_ctzll(n)), i);
    const E6 common = e6_mul_base(e6_sub(e6_pow(zeta, n), e6_one()), inv(to_mont((uint32_t)n)));
    return e6_mul(e6_mul_base(common, wi), e6_inv(e6_sub(zeta, e6_base(wi))));
  }
  void check_air() {
    for (size_t t = 0; t < lay.trees.size(); t++) {
      const auto& T = lay.trees[t];
      for (size_t g = 0; g < T.groups.size(); g++) {
        const auto& G = T.groups[g];
        for (size_t i = 0; i < G.bcols.size(); i++) {
          const auto& vals = cv[t][g][i];
          if (T.air) { chunk_at[{G.module, G.bcols[i]}] = vals[0]; continue; }
          auto sh = shifts_of(t, G.bcols[i]);
          for (size_t k = 0; k < sh.size(); k++) col_at[{G.bcols[i], sh[k]}] = vals[k];
        }
        for (size_t i = 0; i < G.ecols.size(); i++) {
          const auto& vals = cv[t][g][ext_index(t, g, i)];
          if (T.air) { chunk_at[{G.module, G.ecols[i]}] = vals[0]; continue; }
          auto sh = shifts_of(t, G.ecols[i]);
          for (size_t k = 0; k < sh.size(); k++) col_at[{G.ecols[i], sh[k]}] = vals[k];
        }
      }
    }
    const auto& nodes = lay.pg.nodes;
    for (uint32_t m : lay.mod_order) {
      if (lay.fold_root[m] < 0) continue;
      const int64_t n = (int64_t)mod_n(m);
      std::vector<char> seen(nodes.size(), 0);
      lay.collect((uint32_t)lay.fold_root[m], seen);
      std::vector<E6> v(nodes.size());
      for (uint32_t id = 0; id < nodes.size(); id++) {  // children precede parents
        if (!seen[id]) continue;
        const Node& x = nodes[id];
        switch (x.op) {
          case OP_COL: {
            const Column& col = lay.pg.columns[x.a];
            const int s = (int)((((int64_t)(int32_t)x.b) % n + n) % n);
            if (col.kind == KIND_LAGRANGE) {
              const int64_t row = (int64_t)lay.lagrange_row(x.a);
              v[id] = lagrange_at((size_t)n, (size_t)(((row - s) % n + n) % n));
            } else {
              auto it = col_at.find({x.a, s});
              if (it == col_at.end()) reject("no claimed value for column " + col.name);
              v[id] = it->second;
            }
            break;
          }
          case OP_COIN: v[id] = coins.at(x.a); break;
          case OP_CONST: v[id] = e6_base(to_mont(x.a % P)); break;
          case OP_EXPAVG: v[id] = e6_mul_base(exposed.at(x.a), inv(to_mont((uint32_t)n))); break;
          case OP_EXPVAL: v[id] = exposed.at(x.a); break;
          case OP_ADD: v[id] = e6_add(v[x.a], v[x.b]); break;
          case OP_SUB: v[id] = e6_sub(v[x.a], v[x.b]); break;
          default: v[id] = e6_mul(v[x.a], v[x.b]); break;
        }
      }
      const E6 zn = e6_pow(zeta, (uint64_t)n);
      E6 q = e6_zero(), zp = e6_one();
      for (uint32_t i = 0;; i++) {
        auto it = chunk_at.find({m, i});
        if (it == chunk_at.end()) break;
        q = e6_add(q, e6_mul(zp, it->second));
        zp = e6_mul(zp, zn);
      }
      if (!e6_eq(v[lay.fold_root[m]], e6_mul(e6_sub(zn, e6_one()), q)))
        reject("AIR relation check failed for module " + lay.pg.modules[m].name);
    }
  }

  // ------------------------------------------------------------ PCS
  std::vector<uint32_t> classes;
  struct Level { uint32_t module; size_t d; int intro; };
  std::vector<Level> levels;
  std::vector<size_t> level_of;
  int r0 = 0;
  std::vector<uint64_t> pos;
  // device job data
  std::vector<uint32_t> words, shapes;
  std::vector<VerifyJob> pjobs;
  std::vector<std::string> pjob_what;

  static int lg2(uint64_t x) { int k = 0; while ((1ull << k) < x) k++; return k; }
  uint64_t push_words(const uint32_t* p, size_t n) {
    uint64_t o = words.size();
    words.insert(words.end(), p, p + n);
    return o;
  }
  uint64_t push_digests(const std::vector<Digest>& ds) {
    uint64_t o = words.size();
    for (auto& d : ds) words.insert(words.end(), d.v, d.v + 8);
    return o;
  }
  // a Merkle job; groups: (lo words, hi words, nb, ne, log2 pair width)
  // (the rows stay where the decoder put them; they are copied once, here)
  struct JGroup { const uint32_t* lo; const uint32_t* hi; uint32_t nb, ne, logw; };
  std::vector<uint64_t> last_rows;  // word offset of each group's lo row in the last job
  DBufP words_d;                    // `words` on the device (path jobs, then the bridge)
  void add_path_job(const std::vector<JGroup>& gs, const VPath& p, const std::vector<Digest>* inj, const Digest& root,
                    const std::string& what) {
    if (gs.size() > VJ_MAX_GROUPS) reject("too many injected groups");
    VerifyJob J{};
    J.rows_off = words.size();
    last_rows.clear();
    for (auto& g : gs) {
      const size_t w = g.nb + 6 * (size_t)g.ne;
      last_rows.push_back(words.size());
      words.insert(words.end(), g.lo, g.lo + w);
      words.insert(words.end(), g.hi, g.hi + w);
    }
    J.sib_off = push_digests(p.sib);
    J.inj_off = inj && !inj->empty() ? push_digests(*inj) : ~0ull;
    J.root_off = push_words(root.v, 8);
    J.shape_off = (uint32_t)shapes.size();
    for (auto& g : gs) shapes.insert(shapes.end(), {g.nb, g.ne, g.logw});
    J.n_groups = (uint32_t)gs.size();
    J.leaf_idx = p.leaf_idx;
    J.depth = (uint32_t)p.sib.size();
    pjobs.push_back(J);
    pjob_what.push_back(what);
  }

  void pcs_verify() {
    for (uint32_t m : lay.mod_order) {
      bool has = false;
      for (auto& t : lay.trees) for (auto& g : t.groups) if (g.module == m) has = true;
      if (has) classes.push_back(m);
    }
    if (classes.empty()) reject("nothing committed");
    Transcript& fs = lay.fs;
    fs.add("alpha_DEEP");
    for (uint32_t m : classes)
      for (size_t t = 0; t < lay.trees.size(); t++)
        for (size_t g = 0; g < lay.trees[t].groups.size(); g++) {
          if (lay.trees[t].groups[g].module != m) continue;
          for (auto& vals : cv[t][g]) for (auto& v : vals) fs.bind("alpha_DEEP", v.c, 6);
        }
    alpha = digest_e6(fs.compute("alpha_DEEP"));
    std::vector<size_t> idx(classes.size());
    for (size_t i = 0; i < idx.size(); i++) idx[i] = i;
    std::stable_sort(idx.begin(), idx.end(), [&](size_t a, size_t b) { return mod_n(classes[a]) > mod_n(classes[b]); });
    level_of.assign(classes.size(), 0);
    for (size_t l = 0; l < idx.size(); l++) {
      const size_t d = mod_n(classes[idx[l]]);
      levels.push_back({classes[idx[l]], d, MAX_LOG_MODULE - lg2(d)});
      level_of[idx[l]] = l;
    }
    fri_verify();
    c.phase("verify: FRI queries");
    point_samplings();
    c.phase("verify: opening jobs");
    run_path_jobs();
    c.phase("verify: Merkle openings (GPU)");
    bridge();
    c.phase("verify: DEEP bridge");
  }

  void fri_verify() {
    Transcript& fs = lay.fs;
    const int NR = MAX_LOG_MODULE;
    const size_t L = levels.size();
    r0 = levels[0].intro;
    if (r0 >= NR) reject("FRI: first level too small");
    if (fri_roots.size() != (size_t)(NR - 1 - r0)) reject("FRI: wrong number of layer roots");
    if (fq.size() != nq) reject("FRI: wrong number of queries");
    for (auto& q : fq) if (q.size() != (size_t)(NR - r0)) reject("FRI: wrong number of query layers");
    if (lq.size() != L - 1) reject("FRI: wrong number of level query sets");
    for (auto& s : lq) if (s.size() != nq) reject("FRI: wrong number of level queries");
    if (final_field != 1 || final_poly.empty()) reject("FRI: final polynomial must be a non-empty extension vector");
    for (size_t l = 1; l < L; l++) fs.add("fri_level_" + std::to_string(l) + "_gamma");
    for (int j = 0; j < NR; j++) fs.add("fri_fold_" + std::to_string(j));
    for (uint32_t k = 0; k < nq; k++) fs.add("fri_query_" + std::to_string(k));
    std::vector<E6> gam(L);
    for (size_t l = 1; l < L; l++) {
      const std::string nm = "fri_level_" + std::to_string(l) + "_gamma";
      if (l == 1) fs.bind(nm, levels_root.v, 8);
      gam[l] = digest_e6(fs.compute(nm));
    }
    Digest zero{};
    for (int j = 0; j < r0; j++) {
      fs.bind("fri_fold_" + std::to_string(j), zero.v, 8);
      fs.compute("fri_fold_" + std::to_string(j));
    }
    std::vector<Digest> fr(NR);
    std::vector<E6> alphas(NR);
    for (int j = r0; j < NR; j++) {
      fr[j] = j == r0 ? levels_root : fri_roots[j - r0 - 1];
      const std::string nm = "fri_fold_" + std::to_string(j);
      fs.bind(nm, fr[j].v, 8);
      alphas[j] = digest_e6(fs.compute(nm));
    }
    {
      std::vector<uint32_t> fin = {to_mont(0x45585450u), to_mont((uint32_t)final_poly.size())};
      for (auto& v : final_poly) fin.insert(fin.end(), v.c, v.c + 6);
      fs.bind("fri_query_0", fin.data(), fin.size());
    }
    std::map<int, std::vector<size_t>> at_round;
    for (size_t l = 1; l < L; l++) at_round[levels[l].intro].push_back(l);
    const uint32_t inv2 = inv(to_mont(2));
    pos.assign(nq, 0);
    for (uint32_t k = 0; k < nq; k++) {
      const Digest ch = fs.compute("fri_query_" + std::to_string(k));
      const uint64_t s = (((uint64_t)from_mont(ch.v[0]) << 31) ^ (uint64_t)from_mont(ch.v[1])) % (1ull << LOG_N_FRI);
      if (k + 1 < nq) fs.bind("fri_query_" + std::to_string(k + 1), ch.v, 8);
      const auto& Q = fq[k];
      for (int j = r0; j < NR; j++) {
        const VLayer& layer = Q[j - r0];
        const uint64_t row = s >> j, lo = row & ~1ull;
        const size_t nj = (size_t)1 << (LOG_N_FRI - j);
        if (layer.field != 1) reject("FRI: query layer is not an extension layer");
        if (layer.row != row) reject("FRI: query row differs from the transcript's");
        if (layer.path.leaf_idx != lo / 2) reject("FRI: path opens the wrong pair");
        std::vector<JGroup> gs = {{layer.p.c, layer.q.c, 0, 1, (uint32_t)(LOG_N_FRI - j - 1)}};
        if (j == r0) {  // levels tree: every other level's pair is an injection
          for (size_t l = 1; l < L; l++) {
            const VLayer& ld = lq[l - 1][k];
            if (ld.field != 1) reject("FRI: level query is not an extension layer");
            if (ld.path.leaf_idx || !ld.path.sib.empty() || !ld.path.inj.empty()) reject("FRI: level query carries a path");
            if (ld.row != (s >> levels[l].intro)) reject("FRI: level query row differs from the transcript's");
            gs.push_back({ld.p.c, ld.q.c, 0, 1, (uint32_t)lg2((levels[l].d << RATE_LOG) / 2)});
          }
          if (!layer.path.inj.empty()) reject("FRI: levels path carries injection leaves");
          add_path_job(gs, layer.path, nullptr, fr[j], "FRI levels tree at query " + std::to_string(k));
        } else {
          if (!layer.path.inj.empty()) reject("FRI: layer path carries injection leaves");
          add_path_job(gs, layer.path, nullptr, fr[j], "FRI layer " + std::to_string(j) + " at query " + std::to_string(k));
        }
        E6 p = layer.p, q = layer.q;
        if (j == r0)
          for (size_t l : at_round[r0]) {
            p = e6_add(p, e6_mul(lq[l - 1][k].p, gam[l]));
            q = e6_add(q, e6_mul(lq[l - 1][k].q, gam[l]));
          }
        const uint32_t xinv = mont_pow(inv(root_of_unity_mont(LOG_N_FRI - j)), bitrev32((uint32_t)(lo >> 1), lg2(nj / 2)));
        E6 expected = e6_add(e6_mul_base(e6_add(p, q), inv2), e6_mul(e6_mul_base(e6_mul_base(e6_sub(p, q), inv2), xinv), alphas[j]));
        if (j < NR - 1) {
          const uint64_t nrow = row >> 1;
          const bool leaf_p = (nrow & 1) == 0;
          auto it = at_round.find(j + 1);
          if (it != at_round.end())
            for (size_t l : it->second) {
              const VLayer& ld = lq[l - 1][k];
              if (ld.row != nrow) reject("FRI: level query row differs at its intro round");
              expected = e6_add(expected, e6_mul(leaf_p ? ld.p : ld.q, gam[l]));
            }
          if (!e6_eq(expected, leaf_p ? Q[j + 1 - r0].p : Q[j + 1 - r0].q)) reject("FRI: fold mismatch at round " + std::to_string(j + 1));
        } else {
          const uint64_t f = s >> NR;
          if (f >= final_poly.size() || !e6_eq(expected, final_poly[f])) reject("FRI: folded value does not match the final polynomial");
        }
      }
      pos[k] = (uint64_t)Q[0].row << r0;
    }
  }

  // per tree: groups in decreasing row count, ties in declaration order
  // (the leaf level first, then the injected groups), and each group's place
  std::vector<std::vector<size_t>> inj_ord, inj_at;
  void injection_orders() {
    for (const auto& T : lay.trees) {
      std::vector<size_t> o(T.groups.size()), at(T.groups.size());
      for (size_t i = 0; i < o.size(); i++) o[i] = i;
      std::stable_sort(o.begin(), o.end(), [&](size_t a, size_t b) { return mod_n(T.groups[a].module) > mod_n(T.groups[b].module); });
      for (size_t i = 0; i < o.size(); i++) at[o[i]] = i;
      inj_ord.push_back(o);
      inj_at.push_back(at);
    }
  }

  std::vector<std::vector<std::vector<uint64_t>>> row_off;  // query, tree, place in injection order -> lo row
  void point_samplings() {
    if (ps.size() != nq) reject("point samplings: wrong number of queries");
    row_off.assign(nq, std::vector<std::vector<uint64_t>>(lay.trees.size()));
    for (uint32_t k = 0; k < nq; k++) {
      if (ps[k].size() != lay.trees.size()) reject("point samplings: wrong number of batches");
      for (size_t t = 0; t < lay.trees.size(); t++) {
        const VSample& sp = ps[k][t];
        const auto& G = lay.trees[t].groups;
        const std::vector<size_t>& ord = inj_ord[t];
        if (sp.inj.size() != ord.size() - 1) reject("point samplings: wrong number of injected groups");
        auto width_ok = [&](const VRow& r, const Prover::Group& g) { return r.nb == g.bcols.size() && r.ne == g.ecols.size(); };
        if (!width_ok(sp.top_lo, G[ord[0]]) || !width_ok(sp.top_hi, G[ord[0]])) reject("point samplings: top row width");
        const size_t top_rows = mod_n(G[ord[0]].module) << RATE_LOG;
        const uint64_t tlo = (pos[k] >> (LOG_N_FRI - lg2(top_rows))) & ~1ull;
        if (sp.path.leaf_idx != tlo / 2) reject("point samplings: path opens the wrong pair");
        if (sp.path.sib.size() != (size_t)lg2(top_rows / 2)) reject("point samplings: path depth");
        if (!sp.path.inj.empty() && sp.path.inj.size() != ord.size() - 1) reject("point samplings: injection leaves count");
        std::vector<JGroup> gs = {{sp.top_lo.w.data(), sp.top_hi.w.data(), sp.top_lo.nb, sp.top_lo.ne, (uint32_t)lg2(top_rows / 2)}};
        for (size_t i = 1; i < ord.size(); i++) {
          const auto& rows = sp.inj[i - 1];
          if (!width_ok(rows.first, G[ord[i]]) || !width_ok(rows.second, G[ord[i]])) reject("point samplings: injected row width");
          const size_t rws = mod_n(G[ord[i]].module) << RATE_LOG;
          // the injected pair sits on the path: its index is the path index at its width
          const uint64_t lo = (pos[k] >> (LOG_N_FRI - lg2(rws))) & ~1ull;
          if ((sp.path.leaf_idx >> (lg2(top_rows / 2) - lg2(rws / 2))) != lo / 2) reject("point samplings: injected pair off the path");
          gs.push_back({rows.first.w.data(), rows.second.w.data(), rows.first.nb, rows.first.ne, (uint32_t)lg2(rws / 2)});
        }
        add_path_job(gs, sp.path, &sp.path.inj, roots[t], "batch " + std::to_string(t) + " at query " + std::to_string(k));
        row_off[k][t] = last_rows;
      }
    }
  }

  void run_path_jobs() {
    if (pjobs.empty()) return;
    words_d = upload_vec(c, words);
    auto& wd = words_d;
    auto sd = upload_vec(c, shapes), jd = upload_vec(c, pjobs);
    auto bad = std::make_shared<DBuf>(pjobs.size(), c.stream);
    c.timed("verify_paths", 0, 0, [&] {
      k_verify_paths<<<(unsigned)((pjobs.size() + 63) / 64), 64, 0, c.stream>>>((const VerifyJob*)jd->p, (uint32_t)pjobs.size(),
                                                                                 wd->p, sd->p, bad->p);
      LG_LAUNCH();
    });
    std::vector<uint32_t> h(pjobs.size());
    uint32_t* st = c.host_staging(h.size());
    c.d2h(st, bad->p, h.size());
    for (size_t i = 0; i < h.size(); i++)
      if (st[i]) reject(std::string(st[i] == 2 ? "injection leaf mismatch in " : "Merkle path does not authenticate: ") + pjob_what[i]);
  }

  void bridge() {
    // per class: its polynomials (tree, group, base/ext, index), in the
    // alpha order of the DEEP quotient (internal/fri/deep.go:71-111)
    std::vector<E6> cvs, zss, scales;
    std::vector<BridgeTerm> terms;
    std::vector<BridgeJob> jobs;
    struct PolyRef { size_t t, g; bool ext; size_t i; uint32_t scale; std::vector<int> shifts; uint32_t cv0; };
    std::vector<std::vector<PolyRef>> per_class(classes.size());
    std::vector<std::map<int, uint32_t>> z_index(classes.size());
    for (size_t ci = 0; ci < classes.size(); ci++) {
      const uint32_t m = classes[ci];
      const uint32_t w = root_of_unity_mont(lg2(mod_n(m)));
      E6 run = e6_one();
      for (size_t t = 0; t < lay.trees.size(); t++)
        for (size_t g = 0; g < lay.trees[t].groups.size(); g++) {
          const auto& G = lay.trees[t].groups[g];
          if (G.module != m) continue;
          auto add = [&](bool ext, size_t i, uint32_t col) {
            PolyRef pr{t, g, ext, i, (uint32_t)scales.size(), shifts_of(t, col), (uint32_t)cvs.size()};
            scales.push_back(run);
            run = e6_mul(run, alpha);
            const auto& vals = cv[t][g][ext ? ext_index(t, g, i) : i];
            cvs.insert(cvs.end(), vals.begin(), vals.end());
            for (int s : pr.shifts)
              if (!z_index[ci].count(s)) {
                z_index[ci][s] = (uint32_t)zss.size();
                zss.push_back(e6_mul_base(zeta, mont_pow(w, (uint64_t)s)));
              }
            per_class[ci].push_back(pr);
          };
          for (size_t i = 0; i < G.bcols.size(); i++) add(false, i, G.bcols[i]);
          for (size_t i = 0; i < G.ecols.size(); i++) add(true, i, G.ecols[i]);
        }
    }
    for (uint32_t k = 0; k < nq; k++)
      for (size_t ci = 0; ci < classes.size(); ci++) {
        const uint32_t m = classes[ci];
        const size_t rat = mod_n(m) << RATE_LOG;
        const uint64_t lo = (pos[k] >> (LOG_N_FRI - lg2(rat))) & ~1ull;
        BridgeJob J{};
        J.x = mont_pow(root_of_unity_mont(lg2(rat)), bitrev32((uint32_t)lo, lg2(rat)));
        J.t0 = (uint32_t)terms.size();
        for (const PolyRef& pr : per_class[ci]) {
          const size_t at = inj_at[pr.t][pr.g];
          const VSample& sp = ps[k][pr.t];
          const VRow& rlo = at == 0 ? sp.top_lo : sp.inj[at - 1].first;
          const uint64_t width = rlo.nb + 6 * (uint64_t)rlo.ne;
          const uint64_t lo_off = row_off[k][pr.t][at] + (pr.ext ? rlo.nb + 6 * pr.i : pr.i), hi_off = lo_off + width;
          for (size_t q = 0; q < pr.shifts.size(); q++)
            terms.push_back(BridgeTerm{lo_off, hi_off, pr.ext ? 1u : 0u, pr.cv0 + (uint32_t)q, z_index[ci][pr.shifts[q]], pr.scale});
        }
        J.t1 = (uint32_t)terms.size();
        const size_t l = level_of[ci];
        const VLayer& want = l == 0 ? fq[k][0] : lq[l - 1][k];
        J.want_p = want.p;
        J.want_q = want.q;
        jobs.push_back(J);
      }
    if (!words_d) words_d = upload_vec(c, words);
    auto& wd = words_d;
    auto td = upload_vec(c, terms), jd = upload_vec(c, jobs);
    auto cd = upload_vec(c, cvs), zd = upload_vec(c, zss), scd = upload_vec(c, scales);
    auto bad = std::make_shared<DBuf>(jobs.size(), c.stream);
    c.timed("verify_bridge", 0, 0, [&] {
      k_verify_bridge<<<(unsigned)((jobs.size() + 63) / 64), 64, 0, c.stream>>>((const BridgeJob*)jd->p, (uint32_t)jobs.size(),
                                                                                 (const BridgeTerm*)td->p, wd->p, (const E6*)cd->p,
                                                                                 (const E6*)zd->p, (const E6*)scd->p, bad->p);
      LG_LAUNCH();
    });
    uint32_t* st = c.host_staging(jobs.size());
    c.d2h(st, bad->p, jobs.size());
    for (size_t i = 0; i < jobs.size(); i++)
      if (st[i])
        reject("DEEP quotient of module " + lay.pg.modules[classes[i % classes.size()]].name +
               " differs from its FRI level at query " + std::to_string(i / classes.size()));
  }

  void verify(const uint8_t* proof, size_t len, const Digest* setup_root, const char* buses) {
    c.phase_start();
    decode(proof, len);
    c.phase("verify: decode");
    lay.init_order();
    lay.setup_layout();
    injection_orders();
    check_shapes(setup_root);
    derive_challenges();
    check_buses(buses);
    check_air();
    c.phase("verify: transcript and AIR");
    pcs_verify();
  }
};

}  // namespace lg
