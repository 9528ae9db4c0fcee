// CPU oracle (test infrastructure): restatement of loom's prove flow for the
// Poseidon2 backend, from a program descriptor (program.h) and a witness.
// Reference flow: prover/prover.go:142-719; commit
// internal/fri/commitment.go:259-386; quotient
// internal/poly/compute_quotient.go:223-510; open internal/fri/open.go:98-378;
// claimed values internal/fri/values.go:46-110; DEEP
// internal/fri/deep.go:71-266; FRI internal/fri/fri.go:82-736,1024-1272.
#include "prover_core.h"

namespace orc {

// ---------------------------------------------------------------- descriptor
Program parse_program(const uint32_t* w, size_t n) {
  size_t pos = 0;
  auto rd = [&]() -> uint32_t {
    if (pos >= n) throw std::runtime_error("program: truncated");
    return w[pos++];
  };
  auto rds = [&]() {
    uint32_t len = rd();
    std::string s(len, '\0');
    for (uint32_t i = 0; i < len; i += 4) {
      uint32_t x = rd();
      for (uint32_t j = 0; j < 4 && i + j < len; j++) s[i + j] = (char)((x >> (8 * j)) & 0xff);
    }
    return s;
  };
  Program p;
  if (rd() != 0x3150474Cu) throw std::runtime_error("program: bad magic");
  p.n_rounds = rd();
  uint32_t nm = rd(), nc = rd(), nn = rd(), ns = rd();
  for (uint32_t i = 0; i < nm; i++) {
    PModule m;
    m.log_n = rd();
    m.name = rds();
    uint32_t nr = rd();
    for (uint32_t k = 0; k < nr; k++) m.rels.push_back(rd());
    p.modules.push_back(m);
  }
  for (uint32_t i = 0; i < nc; i++) {
    PColumn c;
    c.name = rds();
    c.module = rd(); c.field = rd(); c.kind = rd(); c.param = (int32_t)rd();
    if (c.kind > KIND_SETUP) throw std::runtime_error("program: unknown column kind");
    if (c.module >= nm) throw std::runtime_error("program: column module out of range");
    p.columns.push_back(c);
  }
  for (uint32_t i = 0; i < nn; i++) {
    PNode x; x.op = rd(); x.a = rd(); x.b = rd();
    if (x.op > OP_EXPVAL) throw std::runtime_error("program: unknown node op");
    if (x.op >= OP_ADD && x.op <= OP_MUL && (x.a >= i || x.b >= i))
      throw std::runtime_error("program: node children must precede parents");
    if (x.op == OP_COL && x.a >= nc) throw std::runtime_error("program: node column out of range");
    p.nodes.push_back(x);
  }
  uint32_t n_exposed = 0;
  auto node = [&]() { uint32_t v = rd(); if (v >= nn) throw std::runtime_error("program: step node out of range"); return v; };
  auto column = [&]() { uint32_t v = rd(); if (v >= nc) throw std::runtime_error("program: step column out of range"); return v; };
  for (uint32_t i = 0; i < ns; i++) {
    PStep s;
    s.type = rd();
    s.round = rd();
    if (s.type == STEP_GP || s.type == STEP_RATIO) {
      s.module = rd(); s.num = node(); s.den = node(); s.out = column();
      if (s.type == STEP_RATIO) s.exposed = n_exposed++;
    } else if (s.type == STEP_MULT) {
      uint32_t a = rd(), b = rd();
      if (!a || !b || a > 4096 || b > 4096) throw std::runtime_error("program: bad multiplicity step");
      for (uint32_t k = 0; k < a; k++) s.src.push_back(node());
      for (uint32_t k = 0; k < b; k++) s.tgt.push_back(node());
      for (uint32_t k = 0; k < b; k++) s.outs.push_back(column());
    } else if (s.type == STEP_MULTW) {
      s.width = rd();
      uint32_t a = rd(), b = rd();
      s.flags = rd();
      if (!s.width || s.width > 8 || !a || !b || a > 4096 || b > 4096 || s.flags > 3)
        throw std::runtime_error("program: bad tuple multiplicity step");
      if (s.flags & 1) for (uint32_t k = 0; k < a; k++) s.sel_s.push_back(node());
      if (s.flags & 2) for (uint32_t k = 0; k < b; k++) s.sel_t.push_back(node());
      for (uint32_t k = 0; k < a * s.width; k++) s.src.push_back(node());
      for (uint32_t k = 0; k < b * s.width; k++) s.tgt.push_back(node());
      for (uint32_t k = 0; k < b; k++) s.outs.push_back(column());
    } else if (s.type == STEP_LOGUP) {
      s.module = rd(); s.out = column();
      uint32_t t = rd();
      if (!t || t > 16) throw std::runtime_error("program: bad logup step");
      for (uint32_t k = 0; k < t; k++) { s.e.push_back(node()); s.m.push_back(node()); }
      s.exposed = n_exposed++;
    } else {
      throw std::runtime_error("program: unknown step type");
    }
    if (s.module >= nm) throw std::runtime_error("program: step module out of range");
    p.steps.push_back(s);
  }
  for (const PNode& x : p.nodes)
    if ((x.op == OP_EXPAVG || x.op == OP_EXPVAL) && x.a >= n_exposed)
      throw std::runtime_error("program: exposed value out of range");
  for (uint32_t r = 0; r < p.n_rounds; r++) {
    uint32_t k = rd();
    std::vector<uint32_t> v;
    for (uint32_t i = 0; i < k; i++) v.push_back(rd());
    p.staged.push_back(v);
  }
  return p;
}

std::vector<uint8_t> oracle_prove_bytes(const Program& pg, const uint32_t* const* witness, uint32_t num_queries) {
  Prover p(pg, num_queries);
  return p.prove(witness);
}

Digest oracle_setup_root(const Program& pg, const uint32_t* const* setup) {
  Prover p(pg, 1);
  return p.setup_commit(setup);
}

}  // namespace orc
