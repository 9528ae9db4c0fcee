// The prove as a sequence of device phases, and Prover::prove, which runs
// them with the host transcript.  Order of transcript operations follows
// prover/prover.go:142-719, internal/fri/open.go:98-285 and
// internal/fri/fri.go:606-736.  The phases themselves read no transcript:
// every challenge comes in through set_challenge, so a caller that keeps its
// own transcript (the Go prover through the session entry points of the C
// ABI) drives the same code.
#pragma once
#include "prover.cuh"

namespace lg {

// A committed batch as the openings see it: its groups' base and extension
// polynomial counts in declaration order.
struct OpenBatch {
  const Committed* cm;
  std::vector<uint32_t> nb, ne;
};

// Query openings gathered on the device: row pairs and Merkle paths go to one
// staging buffer (per query, per_q words), then per-query sections are laid
// out in proof order and encoding (big-endian canonical words) by k_assemble
// from a word map, and read back once.
struct OpenPlan {
  std::vector<RowSrc> rows;
  std::vector<PathSrc> paths;
  uint64_t per_q = 0;
  std::vector<uint32_t> map, consts;
  std::vector<PosOp> pops;
  std::vector<SectionSrc> secs;
  uint64_t total = 0;
  size_t start = 0;

  uint64_t add_rows(const uint32_t* lane0, uint64_t stride, uint32_t nl, uint32_t shift) {
    rows.push_back(RowSrc{lane0, stride, nl, shift, per_q});
    uint64_t o = per_q;
    per_q += 2ull * nl;
    return o;
  }
  uint64_t add_path(const TreeDev& t, uint32_t shift, bool with_inj) {
    PathSrc p{};
    p.nodes = t.nodes->p;
    p.inj = with_inj ? (const uint32_t* const*)t.inj_ptrs->p : nullptr;
    p.inj_shift = with_inj ? t.inj_shift->p : nullptr;
    p.log_leaves = t.log_leaves;
    p.n_inj = with_inj ? (uint32_t)t.inj.size() : 0;
    p.shift = shift;
    p.off = per_q;
    paths.push_back(p);
    uint64_t o = per_q;
    per_q += 8ull * (p.log_leaves + p.n_inj);
    return o;
  }
  // section words: constants, the query position (shifted; as a leaf index
  // when `leaf`), copies from the staging buffer
  void begin() { start = map.size(); }
  void konst(uint32_t v) {
    map.push_back((SEC_CONST << 30) | (uint32_t)consts.size());
    consts.push_back(v);
  }
  void posw(uint32_t shift, bool leaf) {
    map.push_back((SEC_POS << 30) | (uint32_t)pops.size());
    pops.push_back(PosOp{shift, leaf ? 1u : 0u});
  }
  void copy(uint64_t off, size_t n) {
    if (off + n > 0x3fffffffu) throw Error(LG_ERR_UNSUPPORTED, "opening block too large");
    for (size_t i = 0; i < n; i++) map.push_back((uint32_t)(off + i));
  }
  SectionSrc end(uint32_t nq) {
    SectionSrc sc{start, total, (uint32_t)(map.size() - start)};
    secs.push_back(sc);
    total += (uint64_t)nq * sc.q_words;
    return sc;
  }

  // The commitment openings of one query (openCommittedAt,
  // internal/fri/open.go:290-378): the batch count, then per batch the row
  // pair of its largest group, that tree's path with its injected leaves,
  // and the row pairs of the other groups (sorted order).
  SectionSrc batches_section(const std::vector<OpenBatch>& bs, uint32_t nq) {
    struct BatchOff { std::vector<uint64_t> rows; uint64_t path; };
    std::vector<BatchOff> boff(bs.size());
    for (size_t b = 0; b < bs.size(); b++) {
      const Committed& cm = *bs[b].cm;
      for (int gi : cm.order) {
        const LdeOut& l = cm.groups[gi];
        uint32_t log_rows = l.log_n + RATE_LOG;
        boff[b].rows.push_back(add_rows(l.lde->p, (size_t)1 << log_rows, l.lanes, (uint32_t)(LOG_N_FRI - log_rows)));
      }
      const LdeOut& top = cm.groups[cm.order[0]];
      boff[b].path = add_path(cm.tree, (uint32_t)(LOG_N_FRI - (top.log_n + RATE_LOG)), true);
    }
    begin();
    konst((uint32_t)bs.size());
    for (size_t b = 0; b < bs.size(); b++) {
      const Committed& cm = *bs[b].cm;
      auto rowpair = [&](int gi, uint64_t off) {
        const LdeOut& l = cm.groups[gi];
        uint32_t nb = bs[b].nb[gi], ne = bs[b].ne[gi];
        if (l.lanes != nb + 6 * ne) throw Error(LG_ERR_INVALID, "opening row width");
        for (int h = 0; h < 2; h++) {
          konst(nb);
          copy(off + (uint64_t)h * l.lanes, nb);
          konst(ne);
          copy(off + (uint64_t)h * l.lanes + nb, 6 * (size_t)ne);
        }
      };
      const LdeOut& top = cm.groups[cm.order[0]];
      rowpair(cm.order[0], boff[b].rows[0]);
      posw((uint32_t)(LOG_N_FRI - (top.log_n + RATE_LOG)), true);
      konst(cm.tree.log_leaves);
      copy(boff[b].path, 8 * (size_t)cm.tree.log_leaves);
      konst((uint32_t)cm.tree.inj.size());
      copy(boff[b].path + 8 * (size_t)cm.tree.log_leaves, 8 * cm.tree.inj.size());
      konst((uint32_t)(cm.order.size() - 1));
      for (size_t s = 1; s < cm.order.size(); s++) rowpair(cm.order[s], boff[b].rows[s]);
    }
    return end(nq);
  }

  // Gathers and lays out every section at the query positions; returns the
  // host copy (the context's pinned staging, valid until its next use).
  const uint32_t* run(Ctx& c, const std::vector<uint32_t>& pos) {
    DBufP asm_d = run_device(c, pos);
    uint32_t* A = c.host_staging(total);
    c.d2h(A, asm_d->p, total);
    return A;
  }
  // The same, left on the device (encoded words, sections at out_off).
  DBufP run_device(Ctx& c, const std::vector<uint32_t>& pos) {
    const uint32_t nq = (uint32_t)pos.size();
    auto pos_d = upload_vec(c, pos);
    auto out_d = std::make_shared<DBuf>(per_q * nq, c.stream);
    {
      auto rd = upload_vec(c, rows);
      uint32_t max_l = 1;
      for (auto& r : rows) max_l = std::max(max_l, r.n_lanes);
      auto pd = upload_vec(c, paths);
      uint32_t max_t = 1;
      for (auto& p : paths) max_t = std::max(max_t, p.log_leaves + p.n_inj);
      c.timed("openings", 8.0 * per_q * nq, 0, [&] {
        if (!rows.empty()) {
          k_gather_rows<<<dim3((max_l + 63) / 64, nq, (unsigned)rows.size()), 64, 0, c.stream>>>(
              (const RowSrc*)rd->p, (uint32_t)rows.size(), pos_d->p, nq, per_q, out_d->p);
          LG_LAUNCH();
        }
        if (!paths.empty()) {
          k_gather_paths<<<dim3((max_t + 31) / 32, nq, (unsigned)paths.size()), 32, 0, c.stream>>>(
              (const PathSrc*)pd->p, pos_d->p, nq, per_q, out_d->p);
          LG_LAUNCH();
        }
        if (per_q) {
          k_proof_words<<<(unsigned)((per_q * nq + 255) / 256), 256, 0, c.stream>>>(out_d->p, per_q * nq);
          LG_LAUNCH();
        }
      });
    }
    auto asm_d = std::make_shared<DBuf>(total, c.stream);
    {
      auto map_d = upload_vec(c, map), consts_d = upload_vec(c, consts);
      auto pops_d = upload_vec(c, pops), secs_d = upload_vec(c, secs);
      uint32_t max_q = 1;
      for (auto& sc : secs) max_q = std::max(max_q, sc.q_words);
      c.timed("openings", 8.0 * total, 0, [&] {
        k_assemble<<<dim3((max_q + 255) / 256, nq, (unsigned)secs.size()), 256, 0, c.stream>>>(
            (const SectionSrc*)secs_d->p, map_d->p, consts_d->p, (const PosOp*)pops_d->p, pos_d->p, out_d->p, per_q, nq,
            asm_d->p);
        LG_LAUNCH();
      });
    }
    return asm_d;
  }
};

struct Prover::OpenPrep {
  OpenPlan op;
  std::vector<SectionSrc> lvl_sec;
  SectionSrc fri_sec{}, batch_sec{};
};

// Length of an encoding, counted without writing (the Writer's methods).
struct Sizer {
  size_t off = 0;
  void u32(uint32_t) { off += 4; }
  void e6(const E6&) { off += 24; }
  void e6w(const uint32_t*) { off += 24; }
  void dg(const Digest&) { off += 32; }
  void str(const std::string& s) { off += 4 + s.size(); }
};

inline void Prover::begin(const uint32_t* const* witness, bool on_device, bool split_upload) {
  setup(witness, on_device, split_upload);
  coins.assign(pg.n_rounds, e6_zero());
  coin_ready.assign(pg.n_rounds, 0);
  fs_slots = std::make_shared<DBuf>(8 * ((size_t)pg.n_rounds + 2), c.stream);
  LG_CK(cudaMemsetAsync(fs_slots->p, 0, 32 * ((size_t)pg.n_rounds + 2), c.stream));
  dev_fs = false;
  pending_roots.clear();
  pending_coins.clear();
  tree_next = 0;
  // the precommitted setup tree (prover/prover.go:175-229): its root binds
  // to the first challenge and stays out of the proof's commitments
  if (has_setup_tree()) {
    committed.push_back(prog->setup->committed);
    tree_next = 1;
  }
}

inline void Prover::set_challenge(const std::string& name, const uint32_t* d) {
  E6 e = e6_zero();
  for (int k = 0; k < 6; k++) e.c[k] = d[k];
  for (uint32_t r = 0; r < pg.n_rounds; r++)
    if (name == coin_name(r)) {
      coins[r] = e;
      coin_ready[r] = 1;
      c.h2d(fs_slot(r), d, 32);
      return;
    }
  if (name == "__zeta") {
    zeta = e;
    zeta_ready = true;
    c.h2d(fs_slot(pg.n_rounds), d, 32);
    return;
  }
  if (name == "alpha_DEEP") { alpha = e; alpha_ready = true; return; }
  const std::string lp = "fri_level_", fp = "fri_fold_";
  if (name.compare(0, lp.size(), lp) == 0 && name.size() > lp.size() + 6 &&
      name.compare(name.size() - 6, 6, "_gamma") == 0) {
    if (fri_next < 0) throw Error(LG_ERR_INVALID, name + ": the FRI levels are not committed yet");
    const size_t l = std::stoul(name.substr(lp.size(), name.size() - lp.size() - 6));
    if (l < 1 || l >= L) throw Error(LG_ERR_INVALID, "no FRI level for " + name);
    gam[l] = e;
    gam_ready[l] = 1;
    c.h2d(gam_d->p + 8 * l, d, 32);
    return;
  }
  if (name.compare(0, fp.size(), fp) == 0 && name.size() > fp.size()) {
    if (fri_next < 0) throw Error(LG_ERR_INVALID, name + ": the FRI levels are not committed yet");
    const int j = std::stoi(name.substr(fp.size()));
    if (j < r0 || j >= NR) throw Error(LG_ERR_INVALID, name + " has no layer to fold");
    c.h2d(chal->p + 8 * (size_t)j, d, 32);
    chal_ready[j] = 1;
    return;
  }
  throw Error(LG_ERR_INVALID, "unknown challenge " + name);
}

// ---- rounds: steps, commit (prover/prover.go:321-411)
inline bool Prover::commit_round(uint32_t r, Digest* root) {
  if (r >= pg.n_rounds) throw Error(LG_ERR_INVALID, "round out of range");
  need_coins(r);
  // a split upload's late columns: round 0's commitment does not read them,
  // everything after it (round 0's own steps included) may
  bool steps_now = false;
  for (const Step& st : pg.steps) steps_now = steps_now || st.round == r;
  if (r > 0 || steps_now) await_upload();
  run_steps(r);
  bool has = false;
  if (tree_next < trees.size() && !trees[tree_next].air && trees[tree_next].round == (int)r) {
    committed.push_back(commit_tree(trees[tree_next], !dev_fs));
    if (dev_fs) pending_roots.push_back({commitments.size(), committed.size() - 1});
    *root = committed.back().tree.root;  // zeros while pending
    commitments.push_back(*root);
    tree_next++;
    has = true;
  }
  if (dev_fs) {  // the values stay on the device until sync_transcript
    for (const Step& st : pg.steps)
      if (st.round == r && exposes(st.type)) exposed_ready[st.exposed] = 1;
  } else {
    read_exposed(r);
  }
  return has;
}

inline std::vector<E6> Prover::round_exposed(uint32_t r) const {
  std::vector<E6> v;
  for (const Step& st : pg.steps)
    if (st.round == r && exposes(st.type)) v.push_back(exposed[st.exposed]);
  return v;
}

// ---- AIR quotients and their commitment (prover/prover.go:461-561)
inline bool Prover::commit_quotient(Digest* root) {
  need_coins(pg.n_rounds);
  await_upload();
  if (tree_next < trees.size() && !trees[tree_next].air)
    throw Error(LG_ERR_INVALID, "the rounds are not all committed yet");
  quotient_all();
  if (tree_next < trees.size() && trees[tree_next].air) {
    committed.push_back(commit_tree(trees[tree_next], !dev_fs));
    if (dev_fs) pending_roots.push_back({commitments.size(), committed.size() - 1});
    *root = committed.back().tree.root;
    commitments.push_back(*root);
    tree_next++;
    return true;
  }
  return false;
}

// ---- claimed values P(zeta w^s) from coefficients (internal/fri/values.go:46-110)
inline void Prover::claimed_values() {
  if (!zeta_ready) throw Error(LG_ERR_INVALID, "challenge __zeta has not been set");
  if (tree_next != trees.size()) throw Error(LG_ERR_INVALID, "the quotient is not committed yet");
  polys.assign(trees.size(), {});
  for (size_t t = 0; t < trees.size(); t++) {
    polys[t].resize(trees[t].groups.size());
    for (size_t g = 0; g < trees[t].groups.size(); g++) {
      const Group& G = trees[t].groups[g];
      size_t n = mod_n(G.module);
      uint32_t lw = root_ext[G.module] ? 6 : 1;
      auto add_poly = [&](uint32_t idx, bool ext) {
        Poly p{t, g, ext, nullptr, pg.modules[G.module].log_n, {}};
        if (trees[t].air) { p.coef = chunk_coef.at(G.module)->p + (size_t)idx * lw * n; p.shifts = {0}; }
        else {
          p.coef = col_coef.at(idx);
          auto it = col_shifts.find(idx);
          if (it != col_shifts.end()) p.shifts = it->second;
        }
        polys[t][g].push_back(p);
      };
      for (uint32_t x : G.bcols) add_poly(x, false);
      for (uint32_t x : G.ecols) add_poly(x, true);
    }
  }
  std::map<std::pair<uint32_t, int>, DBufP> zp;  // (log n, shift) -> powers of zeta w^shift
  std::vector<DotJob> jobs;
  for (auto& pt : polys)
    for (auto& pgp : pt)
      for (auto& p : pgp)
        for (int s : p.shifts) {
          auto key = std::make_pair(p.logn, s);
          if (!zp.count(key)) {
            uint32_t n = 1u << p.logn;
            // zeta w^s with zeta read from its device slot
            const uint32_t ws = mont_pow(root_of_unity_mont((int)p.logn), (uint64_t)s);
            auto b = std::make_shared<DBuf>(6 * (size_t)n, c.stream);
            c.timed("claimed_values", 0, 0, [&] {
              k_e6_powers<<<(n + 127) / 128, 128, 0, c.stream>>>(fs_slot(pg.n_rounds), ws, n, b->p);
              LG_LAUNCH();
            });
            zp[key] = b;
          }
          uint32_t n = 1u << p.logn;
          for (uint32_t w = 0; w < (p.ext ? 6u : 1u); w++)
            jobs.push_back(DotJob{p.coef + (size_t)w * n, zp[key]->p, n, (uint32_t)jobs.size()});
        }
  std::vector<uint32_t> dots(6 * jobs.size());
  if (!jobs.empty()) {
    auto jd = upload_vec(c, jobs);
    auto od = std::make_shared<DBuf>(6 * jobs.size(), c.stream);
    c.timed("claimed_values", 0, 0, [&] {
      k_dot<<<(unsigned)jobs.size(), 256, 0, c.stream>>>((const DotJob*)jd->p, od->p);
      LG_LAUNCH();
    });
    // the DEEP denominators depend on zeta alone: forked after the dot
    // products, they run on the side stream while the host reads the claimed
    // values back and hashes them
    launch_deep_den();
    uint32_t* h = c.host_staging(dots.size());
    c.d2h(h, od->p, dots.size());
    memcpy(dots.data(), h, dots.size() * 4);
  }
  cv.assign(trees.size(), {});
  size_t j = 0;
  for (size_t t = 0; t < trees.size(); t++) {
    cv[t].resize(polys[t].size());
    for (size_t g = 0; g < polys[t].size(); g++)
      for (auto& p : polys[t][g]) {
        std::vector<E6> vals;
        for (size_t si = 0; si < p.shifts.size(); si++) {
          E6 v = e6_zero();
          for (uint32_t w = 0; w < (p.ext ? 6u : 1u); w++, j++) {
            E6 d;
            for (int q = 0; q < 6; q++) d.c[q] = dots[6 * j + q];
            E6 basis = e6_zero();
            basis.c[w] = MONT_ONE;
            v = e6_add(v, p.ext ? e6_mul(d, basis) : d);
          }
          vals.push_back(v);
        }
        cv[t][g].push_back(vals);
      }
  }
  classes = deep_class_list();
}

inline std::vector<uint32_t> Prover::deep_class_list() const {
  std::vector<uint32_t> cl;
  for (uint32_t m : mod_order) {
    bool has = false;
    for (auto& t : trees) for (auto& g : t.groups) if (g.module == m) has = true;
    if (has) cl.push_back(m);
  }
  return cl;
}

inline std::vector<uint32_t> Prover::class_point_factors(uint32_t m) const {
  const uint32_t w_n = root_of_unity_mont((int)pg.modules[m].log_n);
  std::vector<uint32_t> ws;
  for (size_t t = 0; t < trees.size(); t++)
    for (size_t g = 0; g < trees[t].groups.size(); g++) {
      if (trees[t].groups[g].module != m) continue;
      for (const Poly& p : polys[t][g])
        for (int sh : p.shifts) {
          const uint32_t f = mont_pow(w_n, (uint64_t)sh);
          if (std::find(ws.begin(), ws.end(), f) == ws.end()) ws.push_back(f);
        }
    }
  if (ws.size() > DEEP_MAX_POINTS) throw Error(LG_ERR_UNSUPPORTED, "too many distinct opening points");
  return ws;
}

inline void Prover::launch_deep_den() {
  const std::vector<uint32_t> cl = deep_class_list();
  std::vector<DenJob> jobs;
  std::vector<size_t> off;
  size_t words = 0;
  uint32_t max_big = 0;
  for (uint32_t m : cl) {
    DenJob j{};
    const std::vector<uint32_t> ws = class_point_factors(m);
    j.n_points = (uint32_t)ws.size();
    for (size_t k = 0; k < ws.size(); k++) j.ws[k] = ws[k];
    j.logn4 = (int)pg.modules[m].log_n + RATE_LOG;
    j.tw = c.twiddles(j.logn4);
    off.push_back(words);
    words += 6 * (size_t)j.n_points << j.logn4;
    max_big = std::max(max_big, 1u << j.logn4);
    jobs.push_back(j);
  }
  deep_den.assign(cl.size(), nullptr);
  if (cl.empty() || !words) return;
  auto all = std::make_shared<DBuf>(words, c.stream);
  for (size_t i = 0; i < jobs.size(); i++) {
    deep_den[i] = dbuf_slice(all, off[i], 6 * (size_t)jobs[i].n_points << jobs[i].logn4);
    jobs[i].den = deep_den[i]->p;
  }
  auto jd = upload_vec(c, jobs);
  // everything the side stream reads (zeta's slot, tables, job list) is
  // ordered before fork_ev on the main stream
  LG_CK(cudaEventRecord(c.fork_ev, c.stream));
  LG_CK(cudaStreamWaitEvent(c.side, c.fork_ev, 0));
  c.timed("deep_den", 24.0 * (double)words / 6, 0, [&] {
    k_deep_den<<<dim3((max_big + 127) / 128, (unsigned)jobs.size()), 128, 0, c.side>>>((const DenJob*)jd->p,
                                                                                      fs_slot(pg.n_rounds));
    LG_LAUNCH();
  }, c.side);
  LG_CK(cudaEventRecord(c.join_ev, c.side));
  den_pending = true;
}

inline std::vector<E6> Prover::claimed_values_bind_order() const {
  std::vector<E6> out;
  for (uint32_t m : classes)
    for (size_t t = 0; t < trees.size(); t++)
      for (size_t g = 0; g < trees[t].groups.size(); g++) {
        if (trees[t].groups[g].module != m) continue;
        for (auto& vals : cv[t][g]) for (auto& v : vals) out.push_back(v);
      }
  return out;
}

// ---- DEEP codewords on the LDE rows (internal/fri/deep.go:71-266)
inline void Prover::deep_codewords() {
  if (cv.empty()) throw Error(LG_ERR_INVALID, "the claimed values are not computed yet");
  if (!alpha_ready) throw Error(LG_ERR_INVALID, "challenge alpha_DEEP has not been set");
  deep.assign(classes.size(), nullptr);
  DBufP deep_all;  // one allocation for every class's codeword
  {
    size_t words = 0;
    for (uint32_t m : classes) words += 6 * (mod_n(m) << RATE_LOG);
    deep_all = std::make_shared<DBuf>(words, c.stream);
  }
  size_t deep_off = 0;
  std::vector<DeepJob> djobs;
  std::vector<DeepBundle> all_bundles;  // every class's bundles, one upload
  std::vector<size_t> bundle_off;
  std::vector<double> dbytes;
  for (size_t ci = 0; ci < classes.size(); ci++) {
    uint32_t m = classes[ci];
    uint32_t logn = pg.modules[m].log_n;
    size_t big = mod_n(m) << RATE_LOG;
    uint32_t w_n = root_of_unity_mont((int)logn);
    DeepJob jb{};
    std::vector<DeepBundle> bundles;
    std::vector<E6> pts;
    std::vector<uint32_t> pts_w;  // their factors w_n^shift (first-use order, as k_deep_den)
    E6 run = e6_one();
    for (size_t t = 0; t < trees.size(); t++)
      for (size_t g = 0; g < trees[t].groups.size(); g++) {
        if (trees[t].groups[g].module != m) continue;
        const LdeOut& l = committed[t].groups[g];
        uint32_t lane = 0;
        for (size_t i = 0; i < polys[t][g].size(); i++) {
          const Poly& p = polys[t][g][i];
          DeepBundle bu{};
          bu.lane0 = l.lde->p + (size_t)lane * big;
          bu.lane_stride = big;
          bu.ext = p.ext;
          bu.scale = run;
          lane += p.ext ? 6 : 1;
          for (size_t si = 0; si < p.shifts.size(); si++) {
            const uint32_t f = mont_pow(w_n, (uint64_t)p.shifts[si]);
            size_t k = 0;
            while (k < pts_w.size() && pts_w[k] != f) k++;
            if (k == pts.size()) {
              if (pts.size() == DEEP_MAX_POINTS) throw Error(LG_ERR_UNSUPPORTED, "too many distinct opening points");
              pts.push_back(e6_mul_base(zeta, f));
              pts_w.push_back(f);
              jb.a[k] = e6_zero();
            }
            jb.a[k] = e6_add(jb.a[k], e6_mul(run, cv[t][g][i][si]));
            bu.mask |= 1u << k;
          }
          bundles.push_back(bu);
          run = e6_mul(run, alpha);
        }
      }
    for (size_t k = 0; k < pts.size(); k++) jb.z[k] = pts[k];
    jb.n_points = (uint32_t)pts.size();
    bundle_off.push_back(all_bundles.size());
    all_bundles.insert(all_bundles.end(), bundles.begin(), bundles.end());
    jb.n_bundles = (uint32_t)bundles.size();
    jb.logn4 = (int)logn + RATE_LOG;
    jb.tw = c.twiddles(jb.logn4);
    deep[ci] = dbuf_slice(deep_all, deep_off, 6 * big);
    deep_off += 6 * big;
    jb.out = deep[ci]->p;
    if (den_pending && ci < deep_den.size() && deep_den[ci]) jb.den = deep_den[ci]->p;
    djobs.push_back(jb);
    double row_bytes = 24.0;
    for (auto& bu : bundles) row_bytes += bu.ext ? 24.0 : 4.0;
    dbytes.push_back(row_bytes * big);
  }
  auto bundles_d = upload_vec(c, all_bundles);
  for (size_t i = 0; i < djobs.size(); i++) djobs[i].bundles = (const DeepBundle*)bundles_d->p + bundle_off[i];
  if (den_pending) {  // join the side stream's denominators
    LG_CK(cudaStreamWaitEvent(c.stream, c.join_ev, 0));
    den_pending = false;
  }
  auto launch_deep = [&](size_t first, size_t count) {
    std::vector<DeepJob> v(djobs.begin() + first, djobs.begin() + first + count);
    uint32_t max_big = 0;
    double bytes = 0;
    for (size_t i = first; i < first + count; i++) { max_big = std::max(max_big, 1u << djobs[i].logn4); bytes += dbytes[i]; }
    auto jd = upload_vec(c, v);
    c.timed("deep", bytes, 0, [&] {
      k_deep<<<dim3((max_big + 127) / 128, (unsigned)count), 128, 0, c.stream>>>((const DeepJob*)jd->p);
      LG_LAUNCH();
    });
  };
  if (c.batched) launch_deep(0, djobs.size());
  else for (size_t i = 0; i < djobs.size(); i++) launch_deep(i, 1);
}

// ---- FRI levels tree (internal/fri/fri.go:294-317,352-365)
inline Digest Prover::commit_levels() {
  if (deep.empty()) throw Error(LG_ERR_INVALID, "nothing to open: the DEEP codewords are not computed");
  std::vector<size_t> class_at(classes.size());
  for (size_t i = 0; i < class_at.size(); i++) class_at[i] = i;
  std::stable_sort(class_at.begin(), class_at.end(), [&](size_t a, size_t b) { return mod_n(classes[a]) > mod_n(classes[b]); });
  L = class_at.size();
  lvl_log.assign(L, 0);
  lvl.assign(L, nullptr);
  for (size_t l = 0; l < L; l++) { lvl_log[l] = pg.modules[classes[class_at[l]]].log_n; lvl[l] = deep[class_at[l]]; }
  NR = MAX_LOG_MODULE;
  r0 = MAX_LOG_MODULE - (int)lvl_log[0];
  levels_tree = TreeDev();
  levels_tree.log_leaves = lvl_log[0] + RATE_LOG - 1;
  levels_tree.nodes = std::make_shared<DBuf>((size_t)16 << levels_tree.log_leaves, c.stream);
  {
    std::vector<LeafGroup> lgs;
    lgs.push_back(leaf_group(lvl[0]->p, 0, 1, lvl_log[0] + RATE_LOG, levels_tree.nodes->p + ((size_t)8 << levels_tree.log_leaves)));
    for (size_t l = 1; l < L; l++) {
      uint32_t lr = lvl_log[l] + RATE_LOG;
      auto lv = std::make_shared<DBuf>((size_t)8 << (lr - 1), c.stream);
      lgs.push_back(leaf_group(lvl[l]->p, 0, 1, lr, lv->p));
      levels_tree.inj.push_back(lv);
      levels_tree.inj_log_w.push_back(lr - 1);
    }
    if (c.batched) launch_leaves(c, lgs);
    else for (auto& g : lgs) launch_leaves(c, {g});
  }
  build_tree(c, levels_tree, !dev_fs);  // dev_fs: the root is read back after the FRI rounds
  gam.assign(L, e6_zero());
  gam_ready.assign(L, 0);
  gam_d = std::make_shared<DBuf>(8 * L, c.stream);
  layers.assign(NR + 1, nullptr);
  ftrees.assign(NR, TreeDev());
  fri_roots.clear();
  chal = std::make_shared<DBuf>((size_t)8 * NR, c.stream);
  chal_ready.assign(NR, 0);
  nj = (size_t)1 << (LOG_N_FRI - r0);
  fri_next = r0;
  return levels_tree.root;
}

// ---- one FRI round: fold layer j (internal/fri/fri.go:1177-1198), then the
// levels that enter at round j + 1 and the next layer's tree
inline bool Prover::fri_fold_round(int j, bool read_root, Digest* next_root, const FsTail* next_fs, bool* fused) {
  if (fri_next < 0) throw Error(LG_ERR_INVALID, "the FRI levels are not committed yet");
  if (j != fri_next) throw Error(LG_ERR_INVALID, "FRI rounds run in order: the next one is fri_fold_" + std::to_string(fri_next));
  if (!chal_ready[j]) throw Error(LG_ERR_INVALID, "challenge fri_fold_" + std::to_string(j) + " has not been set");
  auto jl = [&](size_t l) { return MAX_LOG_MODULE - (int)lvl_log[l]; };
  auto add_levels = [&](int round) {  // running += gamma_l level_l for the levels entering at `round`
    std::vector<AxpyTerm> terms;
    for (size_t l = 1; l < L; l++)
      if (jl(l) == round) {
        if (!gam_ready[l]) throw Error(LG_ERR_INVALID, "challenge fri_level_" + std::to_string(l) + "_gamma has not been set");
        terms.push_back(AxpyTerm{lvl[l]->p, gam_d->p + 8 * l});
      }
    auto axpy = [&](const std::vector<AxpyTerm>& tv) {
      auto td = upload_vec(c, tv);
      c.timed("fri_axpy", 0, 0, [&] {
        k_axpy_e6<<<(unsigned)((nj + 255) / 256), 256, 0, c.stream>>>(running->p, nj, (const AxpyTerm*)td->p,
                                                                       (uint32_t)tv.size());
        LG_LAUNCH();
      });
    };
    if (terms.empty()) return;
    if (c.batched) axpy(terms);
    else for (auto& tm : terms) axpy({tm});
  };
  if (j == r0) {
    layers[j] = lvl[0];
    ftrees[j] = levels_tree;
    running = std::make_shared<DBuf>(6 * nj, c.stream);
    LG_CK(cudaMemcpyAsync(running->p, lvl[0]->p, 6 * nj * 4, cudaMemcpyDeviceToDevice, c.stream));
    add_levels(j);
  }
  auto next = std::make_shared<DBuf>(3 * nj, c.stream);
  const uint32_t* twj = c.twiddles(LOG_N_FRI - j);
  const uint32_t inv2 = inv(to_mont(2));
  c.timed("fri_fold", 36.0 * nj, 0, [&] {
    k_fold<<<(unsigned)((nj / 2 + 255) / 256), 256, 0, c.stream>>>(running->p, nj, chal->p + 8 * (size_t)j, twj, inv2,
                                                                   next->p);
    LG_LAUNCH();
  });
  running = next;
  nj /= 2;
  fri_next = j + 1;
  if (j + 1 >= NR) return false;
  add_levels(j + 1);
  layers[j + 1] = running;
  TreeDev& t = ftrees[j + 1];
  t.log_leaves = (uint32_t)(LOG_N_FRI - (j + 1) - 1);
  t.nodes = std::make_shared<DBuf>((size_t)16 << t.log_leaves, c.stream);
  launch_leaves(c, {leaf_group(running->p, 0, 1, (uint32_t)(LOG_N_FRI - (j + 1)), t.nodes->p + ((size_t)8 << t.log_leaves))});
  const bool f = build_tree(c, t, read_root, next_fs);
  if (fused) *fused = f;
  if (read_root) {
    fri_roots.push_back(t.root);
    *next_root = t.root;
  }
  return true;
}

inline void Prover::fri_tail(int j0, const DBufP& pre_d, const std::vector<uint32_t>& pre_off,
                             const std::vector<uint32_t>& pre_len) {
  if (fri_next != j0 || j0 <= r0 || j0 >= NR) throw Error(LG_ERR_INVALID, "FRI tail out of order");
  auto jl = [&](size_t l) { return MAX_LOG_MODULE - (int)lvl_log[l]; };
  std::vector<FriRound> rr;
  std::vector<AxpyTerm> terms;
  DBufP cur = running;
  std::vector<DBufP> keep;
  size_t n = nj;
  for (int j = j0; j < NR; j++) {
    FriRound R{};
    R.cur = cur->p;
    auto next = std::make_shared<DBuf>(3 * n, c.stream);
    R.next = next->p;
    R.n = n;
    R.tw = c.twiddles(LOG_N_FRI - j);
    R.term_first = (uint32_t)terms.size();
    for (size_t l = 1; l < L; l++)
      if (jl(l) == j + 1) {
        if (!gam_ready[l]) throw Error(LG_ERR_INVALID, "challenge fri_level_" + std::to_string(l) + "_gamma has not been set");
        terms.push_back(AxpyTerm{lvl[l]->p, gam_d->p + 8 * l});
      }
    R.term_count = (uint32_t)terms.size() - R.term_first;
    if (j + 1 < NR) {
      TreeDev& t = ftrees[j + 1];
      t.log_leaves = (uint32_t)(LOG_N_FRI - (j + 1) - 1);
      t.nodes = std::make_shared<DBuf>((size_t)16 << t.log_leaves, c.stream);
      R.nodes = t.nodes->p;
      R.log_leaves = t.log_leaves;
      R.pre_off = pre_off[j + 1];
      R.pre_len = pre_len[j + 1];
      layers[j + 1] = next;
    }
    rr.push_back(R);
    keep.push_back(next);
    cur = next;
    n /= 2;
  }
  auto rd = upload_vec(c, rr);
  auto td = upload_vec(c, terms.empty() ? std::vector<AxpyTerm>(1) : terms);
  double perms = 0;
  for (auto& R : rr) if (R.nodes) perms += 2.0 * (1u << R.log_leaves);
  c.timed("fri_tail", 0, perms, [&] {
    k_fri_tail<<<1, 1024, 0, c.stream>>>((const FriRound*)rd->p, (uint32_t)rr.size(), (uint32_t)j0,
                                          (const AxpyTerm*)td->p, pre_d->p, chal->p, inv(to_mont(2)));
    LG_LAUNCH();
  });
  running = cur;
  nj = n;
  fri_next = NR;
}

inline void Prover::read_final_poly() {
  if (fri_next != NR) throw Error(LG_ERR_INVALID, "the FRI rounds are not all folded yet");
  final_poly.assign(6 * nj, 0);
  uint32_t* h = c.host_staging(6 * nj);
  c.d2h(h, running->p, 6 * nj);
  memcpy(final_poly.data(), h, 6 * nj * 4);
}

// ---- openings: one gather into a staging buffer, one read-back; then the
// canonical encoding (same order as the proof structs)
// The openings' word map (rows, paths, sections) needs only where the
// layers, trees and batches live, not the positions: lg_prove builds it while
// the device finishes the FRI rounds.
inline void Prover::plan_openings() {
  if (fri_next != NR) throw Error(LG_ERR_INVALID, "the FRI rounds are not all folded yet");
  oplan = std::make_shared<OpenPrep>();
  OpenPlan& OP = oplan->op;
  std::vector<SectionSrc>& lvl_sec = oplan->lvl_sec;
  auto jl = [&](size_t l) { return MAX_LOG_MODULE - (int)lvl_log[l]; };
  std::vector<uint64_t> fri_row_off(NR), fri_path_off(NR), lvl_row_off(L);
  for (int j = r0; j < NR; j++) {
    size_t n_j = (size_t)1 << (LOG_N_FRI - j);
    fri_row_off[j] = OP.add_rows(layers[j]->p, n_j, 6, (uint32_t)j);
    fri_path_off[j] = OP.add_path(ftrees[j], (uint32_t)j, false);
  }
  for (size_t l = 1; l < L; l++)
    lvl_row_off[l] = OP.add_rows(lvl[l]->p, (size_t)1 << (lvl_log[l] + RATE_LOG), 6, (uint32_t)jl(l));
  lvl_sec.assign(L, SectionSrc{});
  for (size_t l = 1; l < L; l++) {  // FRI level openings (one section per level)
    OP.begin();
    OP.konst(1);
    OP.posw((uint32_t)jl(l), false);
    OP.copy(lvl_row_off[l], 12);
    OP.konst(0); OP.konst(0); OP.konst(0);
    lvl_sec[l] = OP.end(num_queries);
  }
  OP.begin();  // FRI fold openings
  OP.konst((uint32_t)(NR - r0));
  for (int j = r0; j < NR; j++) {
    OP.konst(1);
    OP.posw((uint32_t)j, false);
    OP.copy(fri_row_off[j], 12);
    OP.posw((uint32_t)j, true);
    OP.konst(ftrees[j].log_leaves);
    OP.copy(fri_path_off[j], 8 * (size_t)ftrees[j].log_leaves);
    OP.konst(0);
  }
  oplan->fri_sec = OP.end(num_queries);
  std::vector<OpenBatch> obs;
  for (size_t b = 0; b < committed.size(); b++) {
    OpenBatch ob{&committed[b], {}, {}};
    for (const Group& G2 : trees[b].groups) {
      ob.nb.push_back((uint32_t)G2.bcols.size());
      ob.ne.push_back((uint32_t)G2.ecols.size());
    }
    obs.push_back(ob);
  }
  oplan->batch_sec = OP.batches_section(obs, num_queries);
}

inline size_t Prover::open_and_encode(const std::vector<uint32_t>& pos, uint8_t* out, size_t out_cap, bool* in_out) {
  if (final_poly.empty()) throw Error(LG_ERR_INVALID, "the FRI final polynomial is not computed yet");
  if (pos.size() != num_queries) throw Error(LG_ERR_INVALID, "one position per query is needed");
  for (uint32_t s : pos)
    if (s >= (1u << LOG_N_FRI)) throw Error(LG_ERR_INVALID, "query position out of range");
  if (!oplan) plan_openings();
  std::shared_ptr<OpenPrep> prep = std::move(oplan);
  OpenPlan& OP = prep->op;
  const std::vector<SectionSrc>& lvl_sec = prep->lvl_sec;
  const SectionSrc fri_sec = prep->fri_sec, batch_sec = prep->batch_sec;
  DBufP asm_d = OP.run_device(c, pos);
  c.phase("openings gather");
  // The encoding in proof order; `section(W, sc)` appends a per-query
  // section of the gathered words.
  auto emit = [&](auto& W, auto section) {
    W.str("poseidon2");
    {  // exposed values by name: name, one entry (index 0, extension kind 1, value)
      std::vector<std::pair<std::string, size_t>> ev;
      for (const Step& st : pg.steps)
        if (exposes(st.type))
          ev.push_back({pg.columns[st.out].name + (st.type == STEP_LOGUP ? "_total" : "_end"), st.exposed});
      std::sort(ev.begin(), ev.end());
      W.u32((uint32_t)ev.size());
      for (auto& e : ev) {
        W.str(e.first);
        W.u32(1);
        W.u32(0);
        W.u32(1);
        W.e6(exposed[e.second]);
      }
    }
    W.u32((uint32_t)commitments.size());
    for (auto& d : commitments) W.dg(d);
    W.u32((uint32_t)trees.size());
    for (size_t t = 0; t < trees.size(); t++) {
      W.u32((uint32_t)trees[t].groups.size());
      for (size_t g = 0; g < trees[t].groups.size(); g++) {
        const Group& G2 = trees[t].groups[g];
        size_t nbp = G2.bcols.size();
        W.u32((uint32_t)nbp);
        for (size_t i = 0; i < nbp; i++) { W.u32((uint32_t)cv[t][g][i].size()); for (auto& v : cv[t][g][i]) W.e6(v); }
        W.u32((uint32_t)G2.ecols.size());
        for (size_t i = nbp; i < cv[t][g].size(); i++) { W.u32((uint32_t)cv[t][g][i].size()); for (auto& v : cv[t][g][i]) W.e6(v); }
      }
    }
    W.dg(levels_tree.root);
    W.u32((uint32_t)(L - 1));
    for (size_t l = 1; l < L; l++) {
      W.u32(num_queries);
      section(W, lvl_sec[l]);
    }
    W.u32((uint32_t)fri_roots.size());
    for (auto& d : fri_roots) W.dg(d);
    W.u32(1);
    W.u32((uint32_t)nj);
    for (size_t i = 0; i < nj; i++) { uint32_t e[6]; for (int w = 0; w < 6; w++) e[w] = final_poly[w * nj + i]; W.e6w(e); }
    W.u32(num_queries);
    section(W, fri_sec);
    W.u32(0);
    W.u32(num_queries);
    section(W, batch_sec);
  };
  const auto sec_bytes = [&](const SectionSrc& sc) { return (size_t)4 * num_queries * sc.q_words; };
  Sizer sz;
  emit(sz, [&](Sizer& S, const SectionSrc& sc) { S.off += sec_bytes(sc); });
  // A caller buffer in page-locked host memory that holds the whole proof
  // takes the sections straight from the device (no staging copy).
  bool pinned = false;
  if (out && out_cap >= sz.off) {
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, out) == cudaSuccess) pinned = at.type == cudaMemoryTypeHost;
    else cudaGetLastError();
  }
  Writer W(c.proof_buf, out, out_cap);
  if (pinned) {
    emit(W, [&](Writer& Wr, const SectionSrc& sc) {
      const size_t n = sec_bytes(sc);
      uint8_t* dst = Wr.claim(n);
      LG_CK(cudaMemcpyAsync(dst, asm_d->p + sc.out_off, n, cudaMemcpyDeviceToHost, c.stream));
    });
  } else {
    uint32_t* A = c.host_staging(OP.total);
    c.d2h(A, asm_d->p, OP.total);
    W.expect(sz.off);
    emit(W, [&](Writer& Wr, const SectionSrc& sc) { Wr.bytes(A + sc.out_off, (size_t)num_queries * sc.q_words); });
  }
  LG_CK(cudaStreamSynchronize(c.stream));
  c.phase("serialize");
  *in_out = W.in_caller_buffer();
  return W.length();
}

// ---- the device transcript
inline bool Prover::fs_queue(FsQueue& q, const std::string& name, const uint32_t* prev_dev, const DevWords& dev,
                             uint32_t* out) {
  const Transcript::Known k = fs.known(name);
  size_t total = k.name.size() + (k.has_prev ? 8 : 0) + k.binds.size();
  for (auto& d : dev) total += d.second;
  if (total > FS_MAX_MSG) return false;
  if (q.words + total > FS_MAX_MSG) fs_launch(q);  // that chain's digests are then in device memory
  uint32_t pos = q.words;
  auto host = [&](const uint32_t* v, size_t n) {
    if (!n) return;
    q.segs.push_back({nullptr, q.consts.size(), (uint32_t)n, pos});
    q.consts.insert(q.consts.end(), v, v + n);
    pos += (uint32_t)n;
  };
  auto device = [&](const uint32_t* p, uint32_t n) {
    q.segs.push_back({p, 0, n, pos});
    pos += n;
  };
  host(k.name.data(), k.name.size());
  if (k.has_prev) {
    if (k.prev_done) {
      host(k.prev.v, 8);
    } else if (prev_dev && !q.chs.empty() && q.chs.back().out == prev_dev) {
      q.chs.back().fwd = (int32_t)pos;  // forwarded from the previous challenge of the chain
      pos += 8;
    } else if (prev_dev) {
      device(prev_dev, 8);
    } else {
      throw Error(LG_ERR_INVALID, "device transcript: the challenge before " + name + " is not computed");
    }
  }
  host(k.binds.data(), k.binds.size());
  for (auto& d : dev) device(d.first, d.second);
  q.chs.push_back(FsChal{q.words, (uint32_t)total, out, -1});
  q.words += (uint32_t)total;
  return true;
}

inline void Prover::fs_launch(FsQueue& q) {
  if (q.chs.empty()) return;
  auto cd = upload_vec(c, q.consts.empty() ? std::vector<uint32_t>{0} : q.consts);
  std::vector<FsSeg> segs;
  for (auto& sg : q.segs) segs.push_back(FsSeg{sg.dev ? sg.dev : cd->p + sg.off, sg.len, sg.moff});
  auto sd = upload_vec(c, segs.empty() ? std::vector<FsSeg>(1) : segs);
  auto hd = upload_vec(c, q.chs);
  c.timed("fs_chain", 0, 0, [&] {
    k_fs_chain<<<1, 32, 0, c.stream>>>((const FsChal*)hd->p, (uint32_t)q.chs.size(), (const FsSeg*)sd->p,
                                       (uint32_t)segs.size());
    LG_LAUNCH();
  });
  q.chs.clear();
  q.segs.clear();
  q.consts.clear();
  q.words = 0;
}

inline void Prover::sync_transcript() {
  const uint32_t R = pg.n_rounds;
  const size_t X = exposed_d ? n_exposed() : 0, np = pending_roots.size();
  uint32_t* h = c.host_staging(8 * np + 6 * X + 8 * ((size_t)R + 1));
  for (size_t i = 0; i < np; i++)
    LG_CK(cudaMemcpyAsync(h + 8 * i, committed[pending_roots[i].tree].tree.nodes->p + 8, 32, cudaMemcpyDeviceToHost,
                          c.stream));
  if (X) LG_CK(cudaMemcpyAsync(h + 8 * np, exposed_d->p, 24 * X, cudaMemcpyDeviceToHost, c.stream));
  uint32_t* slots = h + 8 * np + 6 * X;
  LG_CK(cudaMemcpyAsync(slots, fs_slots->p, 32 * ((size_t)R + 1), cudaMemcpyDeviceToHost, c.stream));
  LG_CK(cudaStreamSynchronize(c.stream));
  for (size_t i = 0; i < np; i++) {
    Digest d;
    memcpy(d.v, h + 8 * i, 32);
    commitments[pending_roots[i].commitment] = d;
    committed[pending_roots[i].tree].tree.root = d;
  }
  for (const Step& st : pg.steps)
    if (exposes(st.type) && exposed_ready[st.exposed] && X)
      for (int w = 0; w < 6; w++) exposed[st.exposed].c[w] = h[8 * np + 6 * st.exposed + w];
  for (const PendingCoin& pc : pending_coins) {
    const std::string nm = pc.round < R ? coin_name(pc.round) : std::string("__zeta");
    if (pc.commitment >= 0) fs.bind(nm, commitments[pc.commitment].v, 8);
    if (pc.round < R)
      for (const E6& e : round_exposed(pc.round)) {  // entry index, then the value
        uint32_t w[7] = {0};
        for (int k = 0; k < 6; k++) w[1 + k] = e.c[k];
        fs.bind(nm, w, 7);
      }
    const Digest d = fs.compute(nm);
    if (memcmp(d.v, slots + 8 * (size_t)pc.round, 32) != 0)
      throw Error(LG_ERR_CUDA, "device and host transcripts disagree at " + nm);
    E6 e;
    for (int k = 0; k < 6; k++) e.c[k] = d.v[k];
    if (pc.round < R) coins[pc.round] = e;
    else zeta = e;
  }
  pending_roots.clear();
  pending_coins.clear();
}

// ---- the whole prove with the host transcript (prover/prover.go:655-719)
inline size_t Prover::prove(const uint32_t* const* witness, bool on_device, uint8_t* out, size_t out_cap,
                            bool* in_out) {
  ArenaScope arena(&c.dev_arena);  // rewound by the next call on the context
  c.phase_start();
  begin(witness, on_device, true);
  c.phase("setup+upload");
  const uint32_t R = pg.n_rounds;
  for (uint32_t r = 0; r < R; r++) fs.add(coin_name(r));
  fs.add("__zeta");
  {
    const std::string first = coin_name(0);
    auto hb = string_to_elements(0x48415348u, "poseidon2");
    fs.bind(first, hb.data(), hb.size());
    std::vector<uint32_t> sz = {to_mont(0x53495a45u), to_mont((uint32_t)mod_order.size())};
    for (uint32_t m : mod_order) sz.push_back(to_mont((uint32_t)mod_n(m)));
    fs.bind(first, sz.data(), sz.size());
  }
  if (has_setup_tree()) fs.bind(coin_name(0), prog->setup->root.v, 8);
  // The round coins and zeta come from the device transcript (k_fs_chain)
  // over the roots and exposed values where the commits left them: the host
  // queues every phase up to the claimed values without waiting for the
  // device, then replays those challenges (sync_transcript).  A message too
  // long for k_fs_chain switches back to the host transcript.
  dev_fs = true;
  FsQueue q;
  auto to_host = [&] {
    if (!dev_fs) return;
    sync_transcript();
    dev_fs = false;
  };
  // ---- rounds: steps, commit, bind root, sample coin (prover/prover.go:360-411)
  // Queued challenges run as one chain right before the first kernel that
  // reads them: a round's steps, the quotient, the claimed values.
  auto round_has_steps = [&](uint32_t r) {
    for (const Step& st : pg.steps) if (st.round == r) return true;
    return false;
  };
  for (uint32_t r = 0; r < R; r++) {
    Digest root;
    const size_t ci = commitments.size();
    if (round_has_steps(r)) fs_launch(q);
    const bool has = commit_round(r, &root);
    if (dev_fs) {
      DevWords dv;
      if (has) dv.push_back({committed.back().tree.nodes->p + 8, 8});
      for (const Step& st : pg.steps)  // exposed values: entry index 0, then six words
        if (st.round == r && exposes(st.type)) {
          dv.push_back({fs_slot(R + 1), 1});
          dv.push_back({exposed_d->p + 6 * (size_t)st.exposed, 6});
        }
      if (fs_queue(q, coin_name(r), r ? fs_slot(r - 1) : nullptr, dv, fs_slot(r))) {
        pending_coins.push_back({r, has ? (int)ci : -1});
        coin_ready[r] = 1;
        c.phase(("round " + std::to_string(r)).c_str());
        continue;
      }
      fs_launch(q);
      to_host();
      if (has) root = commitments[ci];
    }
    if (has) fs.bind(coin_name(r), root.v, 8);
    // BindExposedValues (prover/prover.go:386-396): the round's logup totals
    // in step order, each as its entry index then six elements
    // (board/logup.go:218-225)
    for (const E6& e : round_exposed(r)) {
      uint32_t w[7] = {0};
      for (int k = 0; k < 6; k++) w[1 + k] = e.c[k];
      fs.bind(coin_name(r), w, 7);
    }
    set_challenge(coin_name(r), fs.compute(coin_name(r)).v);
    c.phase(("round " + std::to_string(r)).c_str());
  }
  // ---- AIR quotients and their commitment
  {
    Digest root;
    const size_t ci = commitments.size();
    fs_launch(q);
    const bool has = commit_quotient(&root);
    bool queued = false;
    if (dev_fs) {
      DevWords dv;
      if (has) dv.push_back({committed.back().tree.nodes->p + 8, 8});
      if (fs_queue(q, "__zeta", R ? fs_slot(R - 1) : nullptr, dv, fs_slot(R))) {
        fs_launch(q);
        pending_coins.push_back({R, has ? (int)ci : -1});
        zeta_ready = true;
        queued = true;
      } else {
        to_host();
        if (has) root = commitments[ci];
      }
    }
    if (!queued) {
      if (has) fs.bind("__zeta", root.v, 8);
      set_challenge("__zeta", fs.compute("__zeta").v);
    }
  }
  c.phase("quotient+air commit");
  // ---- claimed values and alpha_DEEP
  claimed_values();
  to_host();  // the claimed values are read back: replay the device's challenges
  dev_fs = true;  // the FRI levels' challenges again come from the device
  c.phase("claimed values");
  fs.add("alpha_DEEP");
  {
    const std::vector<E6> vals = claimed_values_bind_order();
    const size_t ia = fs.at("alpha_DEEP");
    fs.chs[ia].bindings.reserve(6 * vals.size());
    for (const E6& v : vals) fs.bind_at(ia, v.c, 6);
    set_challenge("alpha_DEEP", fs.compute_at(ia).v);
  }
  c.phase("alpha bind");
  deep_codewords();
  c.phase("deep");
  // ---- FRI
  const Digest lroot = commit_levels();
  c.phase("levels tree");
  for (size_t l = 1; l < L; l++) fs.add("fri_level_" + std::to_string(l) + "_gamma");
  for (int j = 0; j < NR; j++) fs.add("fri_fold_" + std::to_string(j));
  for (uint32_t k = 0; k < num_queries; k++) fs.add("fri_query_" + std::to_string(k));
  Digest zero{};
  if (dev_fs) {
    // the level weights and the folds up to the first layer's, chained on
    // the device from the levels root where the tree left it; replayed with
    // the layer roots' challenges after the rounds
    const uint32_t* lroot_d = levels_tree.nodes->p + 8;
    const uint32_t* prev = nullptr;  // alpha_DEEP: on the host
    for (size_t l = 1; l < L; l++) {
      uint32_t* out = gam_d->p + 8 * l;
      if (!fs_queue(q, "fri_level_" + std::to_string(l) + "_gamma", prev,
                    l == 1 ? DevWords{{lroot_d, 8}} : DevWords{}, out))
        throw Error(LG_ERR_UNSUPPORTED, "level weight message too long");
      gam_ready[l] = 1;
      prev = out;
    }
    fold_dev.assign(r0 + 1, 0);
    for (int j = 0; j <= r0; j++) {
      const std::string nm = "fri_fold_" + std::to_string(j);
      if (j < r0) fs.bind(nm, zero.v, 8);
      if (j < r0 && !prev) {  // nothing from the device in the chain yet: the host has it
        fs.compute(nm);
        continue;
      }
      fold_dev[j] = 1;
      uint32_t* out = chal->p + 8 * (size_t)j;
      if (!fs_queue(q, nm, prev, j == r0 ? DevWords{{lroot_d, 8}} : DevWords{}, out))
        throw Error(LG_ERR_UNSUPPORTED, "fold challenge message too long");
      prev = out;
    }
    chal_ready[r0] = 1;
    fs_launch(q);
  } else {
    for (size_t l = 1; l < L; l++) {
      std::string nm = "fri_level_" + std::to_string(l) + "_gamma";
      if (l == 1) fs.bind(nm, lroot.v, 8);
      set_challenge(nm, fs.compute(nm).v);
    }
    for (int j = 0; j < r0; j++) {
      fs.bind("fri_fold_" + std::to_string(j), zero.v, 8);
      fs.compute("fri_fold_" + std::to_string(j));
    }
    const std::string nm = "fri_fold_" + std::to_string(r0);
    fs.bind(nm, lroot.v, 8);
    set_challenge(nm, fs.compute(nm).v);
  }
  // Fold challenges after the first are computed on the device from the
  // layer roots (k_fs_challenge), so the rounds run without a host round
  // trip; the host replays them after the loop and checks every digest.
  std::vector<uint32_t> pre_all;
  std::vector<uint32_t> pre_off(NR), pre_len(NR);
  for (int j = r0 + 1; j < NR; j++) {
    auto pe = string_to_elements(0x46534944u, "fri_fold_" + std::to_string(j));
    if (pe.size() > 48) throw Error(LG_ERR_UNSUPPORTED, "challenge name too long");
    pre_off[j] = (uint32_t)pre_all.size();
    pre_len[j] = (uint32_t)pe.size();
    pre_all.insert(pre_all.end(), pe.begin(), pe.end());
  }
  auto pre_d = upload_vec(c, pre_all.empty() ? std::vector<uint32_t>{0} : pre_all);
  // the rounds whose next layer has at most fri_tail_leaves leaves run in
  // one block (k_fri_tail); 0 leaves them to the per-round launches
  int j_tail = NR;
  if (c.tune.fri_tail_leaves)
    for (int j = r0 + 1; j < NR; j++)
      if (((size_t)1 << (LOG_N_FRI - (j + 1) - 1)) <= c.tune.fri_tail_leaves) { j_tail = j; break; }
  bool fused = false;  // challenge j already hashed by the block that built tree j's top
  for (int j = r0; j < NR; j++) {
    if (j > r0) {
      if (!fused)
        c.timed("fri_challenge", 0, 0, [&] {
          k_fs_challenge<<<1, 32, 0, c.stream>>>(pre_d->p + pre_off[j], pre_len[j], chal->p + 8 * (size_t)(j - 1),
                                                 ftrees[j].nodes->p + 8, chal->p + 8 * (size_t)j);
          LG_LAUNCH();
        });
      chal_ready[j] = 1;
    }
    if (j == j_tail) {
      for (int k = j + 1; k < NR; k++) chal_ready[k] = 1;
      fri_tail(j, pre_d, pre_off, pre_len);
      break;
    }
    Digest unused;
    FsTail ft{};
    if (j + 1 < NR)
      ft = FsTail{pre_d->p + pre_off[j + 1], pre_len[j + 1], chal->p + 8 * (size_t)j, chal->p + 8 * (size_t)(j + 1)};
    fused = false;
    fri_fold_round(j, false, &unused, j + 1 < NR ? &ft : nullptr, &fused);
  }
  plan_openings();  // host work while the device finishes the rounds
  {
    // one read-back: final polynomial, device challenges, layer roots
    const size_t nroot = (size_t)(NR > r0 + 1 ? NR - r0 - 1 : 0);
    uint32_t* h = c.host_staging(6 * nj + 8 * (size_t)NR + 8 * nroot + 8 + 8 * L);
    LG_CK(cudaMemcpyAsync(h, running->p, 6 * nj * 4, cudaMemcpyDeviceToHost, c.stream));
    LG_CK(cudaMemcpyAsync(h + 6 * nj, chal->p, 8 * (size_t)NR * 4, cudaMemcpyDeviceToHost, c.stream));
    for (int j = r0 + 1; j < NR; j++)
      LG_CK(cudaMemcpyAsync(h + 6 * nj + 8 * (size_t)NR + 8 * (size_t)(j - r0 - 1), ftrees[j].nodes->p + 8, 32,
                            cudaMemcpyDeviceToHost, c.stream));
    uint32_t* hl = h + 6 * nj + 8 * (size_t)NR + 8 * nroot;  // levels root, then the level weights
    if (dev_fs) {
      LG_CK(cudaMemcpyAsync(hl, levels_tree.nodes->p + 8, 32, cudaMemcpyDeviceToHost, c.stream));
      LG_CK(cudaMemcpyAsync(hl + 8, gam_d->p, 32 * L, cudaMemcpyDeviceToHost, c.stream));
    }
    LG_CK(cudaStreamSynchronize(c.stream));
    final_poly.assign(6 * nj, 0);
    memcpy(final_poly.data(), h, 6 * nj * 4);
    if (dev_fs) {  // replay the level weights and the folds up to r0
      memcpy(levels_tree.root.v, hl, 32);
      ftrees[r0].root = levels_tree.root;
      auto check = [&](const std::string& nm, const uint32_t* dev) {
        const Digest d = fs.compute(nm);
        if (memcmp(d.v, dev, 32) != 0) throw Error(LG_ERR_CUDA, "device and host transcripts disagree at " + nm);
        return d;
      };
      for (size_t l = 1; l < L; l++) {
        const std::string nm = "fri_level_" + std::to_string(l) + "_gamma";
        if (l == 1) fs.bind(nm, levels_tree.root.v, 8);
        gam[l] = digest_e6(check(nm, hl + 8 + 8 * l));
      }
      for (int j = 0; j <= r0; j++) {
        if (!fold_dev[j]) continue;
        const std::string nm = "fri_fold_" + std::to_string(j);
        if (j == r0) fs.bind(nm, levels_tree.root.v, 8);
        check(nm, h + 6 * nj + 8 * (size_t)j);
      }
      dev_fs = false;
    }
    fri_roots.clear();
    for (int j = r0 + 1; j < NR; j++) {
      Digest root;
      memcpy(root.v, h + 6 * nj + 8 * (size_t)NR + 8 * (size_t)(j - r0 - 1), 32);
      ftrees[j].root = root;
      fri_roots.push_back(root);
      const std::string nm = "fri_fold_" + std::to_string(j);
      fs.bind(nm, root.v, 8);
      Digest d = fs.compute(nm);
      if (memcmp(d.v, h + 6 * nj + 8 * (size_t)j, 32) != 0)
        throw Error(LG_ERR_CUDA, "device and host transcripts disagree at " + nm);
    }
    std::vector<uint32_t> fin = {to_mont(0x45585450u), to_mont((uint32_t)nj)};
    for (size_t i = 0; i < nj; i++) for (int w = 0; w < 6; w++) fin.push_back(final_poly[w * nj + i]);
    fs.bind("fri_query_0", fin.data(), fin.size());
  }
  c.phase("fri rounds");
  std::vector<uint32_t> pos(num_queries);
  const size_t q0 = num_queries ? fs.at("fri_query_0") : 0;  // declared one after another
  for (uint32_t k = 0; k < num_queries; k++) {
    Digest ch = fs.compute_at(q0 + k);
    uint64_t s = (((uint64_t)from_mont(ch.v[0]) << 31) ^ (uint64_t)from_mont(ch.v[1])) % (1ull << LOG_N_FRI);
    pos[k] = (uint32_t)s;
    if (k + 1 < num_queries) fs.bind_at(q0 + k + 1, ch.v, 8);
  }
  c.phase("query challenges");
  return open_and_encode(pos, out, out_cap, in_out);
}

}  // namespace lg
