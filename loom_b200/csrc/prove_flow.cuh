// Prover::prove: the ordered sequence of device phases and transcript steps.
// Order of transcript operations follows prover/prover.go:142-719,
// internal/fri/open.go:98-285 and internal/fri/fri.go:606-736.
#pragma once
#include "prover.cuh"

namespace lg {

inline size_t Prover::prove(const uint32_t* const* witness, bool on_device, uint8_t* out, size_t out_cap,
                            bool* in_out) {
  ArenaScope arena(&c.dev_arena);  // rewound by the next call on the context
  c.phase_start();
  setup(witness, on_device);
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
  // ---- the precommitted setup tree: its root binds to the first challenge
  // and stays out of the proof's commitments (prover/prover.go:175-229)
  size_t ti = 0;
  if (!trees.empty() && trees[0].setup) {
    committed.push_back(prog->setup->committed);
    fs.bind(coin_name(0), prog->setup->root.v, 8);
    ti = 1;
  }
  // ---- rounds: steps, commit, bind root, sample coin (prover/prover.go:360-411)
  coins.assign(R, e6_zero());
  for (uint32_t r = 0; r < R; r++) {
    run_steps(r);
    if (ti < trees.size() && !trees[ti].air && trees[ti].round == (int)r) {
      committed.push_back(commit_tree(trees[ti]));
      Digest root = committed.back().tree.root;
      commitments.push_back(root);
      fs.bind(coin_name(r), root.v, 8);
      ti++;
    }
    // BindExposedValues (prover/prover.go:386-396): the round's logup totals
    // in step order, each as its entry index then six elements
    // (board/logup.go:218-225)
    read_exposed(r);
    for (const Step& st : pg.steps) {
      if (st.round != r || !exposes(st.type)) continue;
      uint32_t w[7] = {0};
      for (int k = 0; k < 6; k++) w[1 + k] = exposed[st.exposed].c[k];
      fs.bind(coin_name(r), w, 7);
    }
    coins[r] = digest_e6(fs.compute(coin_name(r)));
    c.phase(("round " + std::to_string(r)).c_str());
  }
  // ---- AIR quotients and their commitment (prover/prover.go:461-561)
  quotient_all();
  if (ti < trees.size() && trees[ti].air) {
    committed.push_back(commit_tree(trees[ti]));
    Digest root = committed.back().tree.root;
    commitments.push_back(root);
    fs.bind("__zeta", root.v, 8);
    ti++;
  }
  zeta = digest_e6(fs.compute("__zeta"));
  c.phase("quotient+air commit");

  // ---- claimed values P(zeta w^s) from coefficients (internal/fri/values.go:46-110)
  struct Poly { size_t t, g; bool ext; const uint32_t* coef; uint32_t logn; std::vector<int> shifts; };
  std::vector<std::vector<std::vector<Poly>>> polys(trees.size());  // [tree][group] base polys then ext polys
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
  std::map<std::pair<uint32_t, int>, E6> zpoint;
  std::vector<DotJob> jobs;
  for (auto& pt : polys)
    for (auto& pgp : pt)
      for (auto& p : pgp)
        for (int s : p.shifts) {
          auto key = std::make_pair(p.logn, s);
          if (!zp.count(key)) {
            uint32_t n = 1u << p.logn;
            E6 z = e6_mul_base(zeta, mont_pow(root_of_unity_mont((int)p.logn), (uint64_t)s));
            zpoint[key] = z;
            auto b = std::make_shared<DBuf>(6 * (size_t)n, c.stream);
            c.timed("claimed_values", 0, 0, [&] {
              k_e6_powers<<<(n + 127) / 128, 128, 0, c.stream>>>(z, n, b->p);
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
    uint32_t* h = c.host_staging(dots.size());
    c.d2h(h, od->p, dots.size());
    memcpy(dots.data(), h, dots.size() * 4);
  }
  // values[t][g][poly][shift]
  std::vector<std::vector<std::vector<std::vector<E6>>>> cv(trees.size());
  {
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
  }
  // DEEP classes = modules with committed groups, in sorted order
  std::vector<uint32_t> classes;
  for (uint32_t m : mod_order) {
    bool has = false;
    for (auto& t : trees) for (auto& g : t.groups) if (g.module == m) has = true;
    if (has) classes.push_back(m);
  }
  fs.add("alpha_DEEP");
  for (uint32_t m : classes)
    for (size_t t = 0; t < trees.size(); t++)
      for (size_t g = 0; g < trees[t].groups.size(); g++) {
        if (trees[t].groups[g].module != m) continue;
        for (auto& vals : cv[t][g]) for (auto& v : vals) fs.bind("alpha_DEEP", v.c, 6);
      }
  E6 alpha = digest_e6(fs.compute("alpha_DEEP"));
  c.phase("claimed values+bind");

  // ---- DEEP codewords on the LDE rows (internal/fri/deep.go:71-266)
  std::vector<DBufP> deep(classes.size());
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
            E6 z = e6_mul_base(zeta, mont_pow(w_n, (uint64_t)p.shifts[si]));
            size_t k = 0;
            while (k < pts.size() && !e6_eq(pts[k], z)) k++;
            if (k == pts.size()) {
              if (pts.size() == DEEP_MAX_POINTS) throw Error(LG_ERR_UNSUPPORTED, "too many distinct opening points");
              pts.push_back(z);
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
    djobs.push_back(jb);
    double row_bytes = 24.0;
    for (auto& bu : bundles) row_bytes += bu.ext ? 24.0 : 4.0;
    dbytes.push_back(row_bytes * big);
  }
  auto bundles_d = upload_vec(c, all_bundles);
  for (size_t i = 0; i < djobs.size(); i++) djobs[i].bundles = (const DeepBundle*)bundles_d->p + bundle_off[i];
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

  c.phase("deep");
  // ---- FRI (internal/fri/fri.go:352-365,606-736)
  std::vector<size_t> class_at(classes.size());
  for (size_t i = 0; i < class_at.size(); i++) class_at[i] = i;
  std::stable_sort(class_at.begin(), class_at.end(), [&](size_t a, size_t b) { return mod_n(classes[a]) > mod_n(classes[b]); });
  const size_t L = class_at.size();
  if (L == 0) throw Error(LG_ERR_INVALID, "nothing to open");
  std::vector<uint32_t> lvl_log(L);
  std::vector<DBufP> lvl(L);
  for (size_t l = 0; l < L; l++) { lvl_log[l] = pg.modules[classes[class_at[l]]].log_n; lvl[l] = deep[class_at[l]]; }
  const int NR = MAX_LOG_MODULE;
  const int r0 = MAX_LOG_MODULE - (int)lvl_log[0];
  auto jl = [&](size_t l) { return MAX_LOG_MODULE - (int)lvl_log[l]; };
  for (size_t l = 1; l < L; l++) fs.add("fri_level_" + std::to_string(l) + "_gamma");
  for (int j = 0; j < NR; j++) fs.add("fri_fold_" + std::to_string(j));
  for (uint32_t k = 0; k < num_queries; k++) fs.add("fri_query_" + std::to_string(k));
  TreeDev levels_tree;
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
  build_tree(c, levels_tree);
  c.phase("levels tree");
  std::vector<E6> gam(L);
  for (size_t l = 1; l < L; l++) {
    std::string nm = "fri_level_" + std::to_string(l) + "_gamma";
    if (l == 1) fs.bind(nm, levels_tree.root.v, 8);
    gam[l] = digest_e6(fs.compute(nm));
  }
  Digest zero{};
  for (int j = 0; j < r0; j++) {
    fs.bind("fri_fold_" + std::to_string(j), zero.v, 8);
    fs.compute("fri_fold_" + std::to_string(j));
  }
  std::vector<DBufP> layers(NR + 1);
  std::vector<TreeDev> ftrees(NR);
  std::vector<Digest> fri_roots;
  // Fold challenges after the first are computed on the device from the
  // layer roots (k_fs_challenge), so the rounds run without a host round
  // trip; the host replays them after the loop and checks every digest.
  auto chal = std::make_shared<DBuf>((size_t)8 * NR, c.stream);
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
  size_t nj = (size_t)1 << (LOG_N_FRI - r0);
  auto running = std::make_shared<DBuf>(6 * nj, c.stream);
  LG_CK(cudaMemcpyAsync(running->p, lvl[0]->p, 6 * nj * 4, cudaMemcpyDeviceToDevice, c.stream));
  const uint32_t inv2 = inv(to_mont(2));
  for (int j = r0; j < NR; j++) {
    if (j == r0) layers[j] = lvl[0];
    {
      std::vector<AxpyTerm> terms;
      for (size_t l = 1; l < L; l++)
        if (jl(l) == j) terms.push_back(AxpyTerm{lvl[l]->p, gam[l]});
      auto axpy = [&](const std::vector<AxpyTerm>& tv) {
        auto td = upload_vec(c, tv);
        c.timed("fri_axpy", 0, 0, [&] {
          k_axpy_e6<<<(unsigned)((nj + 255) / 256), 256, 0, c.stream>>>(running->p, nj, (const AxpyTerm*)td->p,
                                                                         (uint32_t)tv.size());
          LG_LAUNCH();
        });
      };
      if (!terms.empty()) {
        if (c.batched) axpy(terms);
        else for (auto& tm : terms) axpy({tm});
      }
    }
    if (j > r0) layers[j] = running;
    if (j == r0) {
      ftrees[j] = levels_tree;
      const std::string nm = "fri_fold_" + std::to_string(j);
      fs.bind(nm, levels_tree.root.v, 8);
      Digest d = fs.compute(nm);
      c.h2d(chal->p + 8 * (size_t)j, d.v, 32);
    } else {
      TreeDev& t = ftrees[j];
      t.log_leaves = (uint32_t)(LOG_N_FRI - j - 1);
      t.nodes = std::make_shared<DBuf>((size_t)16 << t.log_leaves, c.stream);
      launch_leaves(c, {leaf_group(running->p, 0, 1, (uint32_t)(LOG_N_FRI - j), t.nodes->p + ((size_t)8 << t.log_leaves))});
      build_tree(c, t, false);
      c.timed("fri_challenge", 0, 0, [&] {
        k_fs_challenge<<<1, 32, 0, c.stream>>>(pre_d->p + pre_off[j], pre_len[j], chal->p + 8 * (size_t)(j - 1),
                                               t.nodes->p + 8, chal->p + 8 * (size_t)j);
        LG_LAUNCH();
      });
    }
    auto next = std::make_shared<DBuf>(3 * nj, c.stream);
    const uint32_t* twj = c.twiddles(LOG_N_FRI - j);
    c.timed("fri_fold", 36.0 * nj, 0, [&] {
      k_fold<<<(unsigned)((nj / 2 + 255) / 256), 256, 0, c.stream>>>(running->p, nj, chal->p + 8 * (size_t)j, twj, inv2,
                                                                     next->p);
      LG_LAUNCH();
    });
    running = next;
    nj /= 2;
  }
  std::vector<uint32_t> final_poly(6 * nj);
  {
    // one read-back: final polynomial, device challenges, layer roots
    const size_t nroot = (size_t)(NR > r0 + 1 ? NR - r0 - 1 : 0);
    uint32_t* h = c.host_staging(6 * nj + 8 * (size_t)NR + 8 * nroot);
    LG_CK(cudaMemcpyAsync(h, running->p, 6 * nj * 4, cudaMemcpyDeviceToHost, c.stream));
    LG_CK(cudaMemcpyAsync(h + 6 * nj, chal->p, 8 * (size_t)NR * 4, cudaMemcpyDeviceToHost, c.stream));
    for (int j = r0 + 1; j < NR; j++)
      LG_CK(cudaMemcpyAsync(h + 6 * nj + 8 * (size_t)NR + 8 * (size_t)(j - r0 - 1), ftrees[j].nodes->p + 8, 32,
                            cudaMemcpyDeviceToHost, c.stream));
    LG_CK(cudaStreamSynchronize(c.stream));
    memcpy(final_poly.data(), h, 6 * nj * 4);
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
  for (uint32_t k = 0; k < num_queries; k++) {
    Digest ch = fs.compute("fri_query_" + std::to_string(k));
    uint64_t s = (((uint64_t)from_mont(ch.v[0]) << 31) ^ (uint64_t)from_mont(ch.v[1])) % (1ull << LOG_N_FRI);
    pos[k] = (uint32_t)s;
    if (k + 1 < num_queries) fs.bind("fri_query_" + std::to_string(k + 1), ch.v, 8);
  }

  c.phase("query challenges");
  // ---- openings: one gather into a staging buffer, one read-back
  std::vector<RowSrc> rows;
  std::vector<PathSrc> paths;
  uint64_t per_q = 0;
  auto add_rows = [&](const uint32_t* lane0, uint64_t stride, uint32_t nl, uint32_t shift) {
    rows.push_back(RowSrc{lane0, stride, nl, shift, per_q});
    uint64_t o = per_q;
    per_q += 2ull * nl;
    return o;
  };
  auto add_path = [&](const TreeDev& t, uint32_t shift, bool with_inj) {
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
  };
  std::vector<uint64_t> fri_row_off(NR), fri_path_off(NR), lvl_row_off(L);
  for (int j = r0; j < NR; j++) {
    size_t n_j = (size_t)1 << (LOG_N_FRI - j);
    fri_row_off[j] = add_rows(layers[j]->p, n_j, 6, (uint32_t)j);
    fri_path_off[j] = add_path(ftrees[j], (uint32_t)j, false);
  }
  for (size_t l = 1; l < L; l++) lvl_row_off[l] = add_rows(lvl[l]->p, (size_t)1 << (lvl_log[l] + RATE_LOG), 6, (uint32_t)jl(l));
  struct BatchOff { std::vector<uint64_t> rows; uint64_t path; };
  std::vector<BatchOff> boff(committed.size());
  for (size_t b = 0; b < committed.size(); b++) {
    const Committed& cm = committed[b];
    for (int gi : cm.order) {
      const LdeOut& l = cm.groups[gi];
      uint32_t log_rows = l.log_n + RATE_LOG;
      boff[b].rows.push_back(add_rows(l.lde->p, (size_t)1 << log_rows, l.lanes, (uint32_t)(LOG_N_FRI - log_rows)));
    }
    const LdeOut& top = cm.groups[cm.order[0]];
    boff[b].path = add_path(cm.tree, (uint32_t)(LOG_N_FRI - (top.log_n + RATE_LOG)), true);
  }
  auto pos_d = upload_vec(c, pos);
  auto out_d = std::make_shared<DBuf>(per_q * num_queries, c.stream);
  {
    auto rd = upload_vec(c, rows);
    uint32_t max_l = 1;
    for (auto& r : rows) max_l = std::max(max_l, r.n_lanes);
    auto pd = upload_vec(c, paths);
    uint32_t max_t = 1;
    for (auto& p : paths) max_t = std::max(max_t, p.log_leaves + p.n_inj);
    c.timed("openings", 8.0 * per_q * num_queries, 0, [&] {
      k_gather_rows<<<dim3((max_l + 63) / 64, num_queries, (unsigned)rows.size()), 64, 0, c.stream>>>(
          (const RowSrc*)rd->p, (uint32_t)rows.size(), pos_d->p, num_queries, per_q, out_d->p);
      LG_LAUNCH();
      k_gather_paths<<<dim3((max_t + 31) / 32, num_queries, (unsigned)paths.size()), 32, 0, c.stream>>>(
          (const PathSrc*)pd->p, pos_d->p, num_queries, per_q, out_d->p);
      LG_LAUNCH();
      k_proof_words<<<(unsigned)((per_q * num_queries + 255) / 256), 256, 0, c.stream>>>(out_d->p,
                                                                                         per_q * num_queries);
      LG_LAUNCH();
    });
  }
  // ---- per-query sections, laid out on the GPU in proof order and encoding
  struct SecBuild {
    std::vector<uint32_t> map, consts;
    std::vector<PosOp> pops;
    std::vector<SectionSrc> secs;
    uint64_t total = 0;
    size_t start = 0;
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
  } SB;
  std::vector<SectionSrc> lvl_sec(L);
  for (size_t l = 1; l < L; l++) {  // FRI level openings (one section per level)
    SB.begin();
    SB.konst(1);
    SB.posw((uint32_t)jl(l), false);
    SB.copy(lvl_row_off[l], 12);
    SB.konst(0); SB.konst(0); SB.konst(0);
    lvl_sec[l] = SB.end(num_queries);
  }
  SB.begin();  // FRI fold openings
  SB.konst((uint32_t)(NR - r0));
  for (int j = r0; j < NR; j++) {
    SB.konst(1);
    SB.posw((uint32_t)j, false);
    SB.copy(fri_row_off[j], 12);
    SB.posw((uint32_t)j, true);
    SB.konst(ftrees[j].log_leaves);
    SB.copy(fri_path_off[j], 8 * (size_t)ftrees[j].log_leaves);
    SB.konst(0);
  }
  const SectionSrc fri_sec = SB.end(num_queries);
  SB.begin();  // batch openings: rows of every group, the batch tree's path
  SB.konst((uint32_t)committed.size());
  for (size_t b = 0; b < committed.size(); b++) {
    const Committed& cm = committed[b];
    auto rowpair = [&](int gi, uint64_t off) {
      const LdeOut& l = cm.groups[gi];
      const Group& G2 = trees[b].groups[gi];
      uint32_t nb = (uint32_t)G2.bcols.size(), ne = (uint32_t)G2.ecols.size();
      if (l.lanes != nb + 6 * ne) throw Error(LG_ERR_INVALID, "opening row width");
      for (int h = 0; h < 2; h++) {
        SB.konst(nb);
        SB.copy(off + (uint64_t)h * l.lanes, nb);
        SB.konst(ne);
        SB.copy(off + (uint64_t)h * l.lanes + nb, 6 * (size_t)ne);
      }
    };
    const LdeOut& top = cm.groups[cm.order[0]];
    rowpair(cm.order[0], boff[b].rows[0]);
    SB.posw((uint32_t)(LOG_N_FRI - (top.log_n + RATE_LOG)), true);
    SB.konst(cm.tree.log_leaves);
    SB.copy(boff[b].path, 8 * (size_t)cm.tree.log_leaves);
    SB.konst((uint32_t)cm.tree.inj.size());
    SB.copy(boff[b].path + 8 * (size_t)cm.tree.log_leaves, 8 * cm.tree.inj.size());
    SB.konst((uint32_t)(cm.order.size() - 1));
    for (size_t s = 1; s < cm.order.size(); s++) rowpair(cm.order[s], boff[b].rows[s]);
  }
  const SectionSrc batch_sec = SB.end(num_queries);
  auto asm_d = std::make_shared<DBuf>(SB.total, c.stream);
  {
    auto map_d = upload_vec(c, SB.map), consts_d = upload_vec(c, SB.consts);
    auto pops_d = upload_vec(c, SB.pops), secs_d = upload_vec(c, SB.secs);
    uint32_t max_q = 1;
    for (auto& sc : SB.secs) max_q = std::max(max_q, sc.q_words);
    c.timed("openings", 8.0 * SB.total, 0, [&] {
      k_assemble<<<dim3((max_q + 255) / 256, num_queries, (unsigned)SB.secs.size()), 256, 0, c.stream>>>(
          (const SectionSrc*)secs_d->p, map_d->p, consts_d->p, (const PosOp*)pops_d->p, pos_d->p, out_d->p, per_q,
          num_queries, asm_d->p);
      LG_LAUNCH();
    });
  }
  uint32_t* A = c.host_staging(SB.total);
  c.d2h(A, asm_d->p, SB.total);

  c.phase("openings gather");
  // ---- canonical encoding (same order as the proof structs)
  Writer W(c.proof_buf, out, out_cap);
  W.expect((size_t)4 * SB.total + (1 << 20));
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
  auto section = [&](const SectionSrc& sc) { W.bytes(A + sc.out_off, (size_t)num_queries * sc.q_words); };
  W.dg(levels_tree.root);
  W.u32((uint32_t)(L - 1));
  for (size_t l = 1; l < L; l++) {
    W.u32(num_queries);
    section(lvl_sec[l]);
  }
  W.u32((uint32_t)fri_roots.size());
  for (auto& d : fri_roots) W.dg(d);
  W.u32(1);
  W.u32((uint32_t)nj);
  for (size_t i = 0; i < nj; i++) { uint32_t e[6]; for (int w = 0; w < 6; w++) e[w] = final_poly[w * nj + i]; W.e6w(e); }
  W.u32(num_queries);
  section(fri_sec);
  W.u32(0);
  W.u32(num_queries);
  section(batch_sec);
  LG_CK(cudaStreamSynchronize(c.stream));
  c.phase("serialize");
  *in_out = W.in_caller_buffer();
  return W.length();
}

}  // namespace lg
