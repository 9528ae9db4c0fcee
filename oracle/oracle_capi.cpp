// C entry points of the CPU oracle (TEST INFRASTRUCTURE ONLY: loaded by
// tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg through
// ctypes; never by the product library).
//
// Field words crossing this interface are Montgomery words (R = 2^32), the
// in-memory layout of gnark-crypto's koalabear.Element, except where a
// function says "canonical".
#include <algorithm>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

#include "oracle.h"
#include "program.h"

namespace orc {
std::vector<uint8_t> oracle_prove_bytes(const Program& pg, const uint32_t* const* witness, uint32_t num_queries);
void oracle_verify_bytes(const Program& pg, const uint8_t* proof, size_t len, uint32_t num_queries, const std::string& buses,
                         const std::vector<Digest>& setup_roots);
Digest oracle_setup_root(const Program& pg, const uint32_t* const* setup);
}
using namespace orc;

static thread_local std::string g_err;

extern "C" {

const char* oracle_last_error() { return g_err.c_str(); }

// The last proof made on this thread, for oracle_last_proof.
static thread_local std::vector<uint8_t> g_last_proof;

// Full prove; proof bytes in the canonical encoding.  Returns 0 on success,
// 1 when *out_len is too small (required size written back; the proof is
// kept for oracle_last_proof), 2 on error.
int oracle_prove(const uint32_t* program, size_t nwords, const uint32_t* const* witness, uint32_t num_queries,
                 uint8_t* out, size_t* out_len) {
  try {
    Program pg = parse_program(program, nwords);
    std::vector<uint8_t> b = oracle_prove_bytes(pg, witness, num_queries);
    if (*out_len < b.size()) {
      *out_len = b.size();
      g_last_proof = std::move(b);
      return 1;
    }
    memcpy(out, b.data(), b.size());
    *out_len = b.size();
    return 0;
  } catch (std::exception& e) {
    g_err = e.what();
    return 2;
  }
}

// Copies out the proof that the last oracle_prove on this thread kept
// because its buffer was too small.  Returns 0, or 1 with the size written
// back when *out_len is still too small.
int oracle_last_proof(uint8_t* out, size_t* out_len) {
  if (*out_len < g_last_proof.size()) { *out_len = g_last_proof.size(); return 1; }
  memcpy(out, g_last_proof.data(), g_last_proof.size());
  *out_len = g_last_proof.size();
  return 0;
}

// Verifies proof bytes against the program (verifier/verifier.go:487-533).
// `buses` (may be NULL) lists the program's product and logup buses as
// "P:end,end;L:total,total,...".  `setup_roots` holds n_setup_roots digests
// (8 canonical words each), the verification key of a program with setup
// columns.  Returns 0 when the proof is accepted, 2 when it is rejected or
// malformed (the reason in oracle_last_error()).
int oracle_verify(const uint32_t* program, size_t nwords, const uint8_t* proof, size_t len, uint32_t num_queries,
                  const char* buses, const uint32_t* setup_roots, uint32_t n_setup_roots) {
  try {
    Program pg = parse_program(program, nwords);
    std::vector<Digest> vk(n_setup_roots);
    for (uint32_t i = 0; i < n_setup_roots; i++) memcpy(vk[i].v, setup_roots + 8 * i, 32);
    oracle_verify_bytes(pg, proof, len, num_queries, buses ? buses : "", vk);
    return 0;
  } catch (std::exception& e) {
    g_err = e.what();
    return 2;
  }
}

// Root of the setup tree (setup/setup.go:68-124) of a program's setup
// columns (Montgomery words, descriptor order), as 8 canonical words.
int oracle_setup(const uint32_t* program, size_t nwords, const uint32_t* const* setup, uint32_t* root_out) {
  try {
    Program pg = parse_program(program, nwords);
    Digest d = oracle_setup_root(pg, setup);
    memcpy(root_out, d.v, 32);
    return 0;
  } catch (std::exception& e) {
    g_err = e.what();
    return 2;
  }
}

// Canonical values in/out.
void oracle_p2_permute(uint32_t* state, int width) { p2_permute(state, width); }

// Round keys as 27 rows of `width` canonical values; partial rows hold their
// one key in column 0 and zeros elsewhere (the zkc constants layout).
int oracle_p2_round_keys(int width, uint32_t* out) {
  auto rk = p2_round_keys(width, 6, 21);
  for (size_t r = 0; r < rk.size(); r++)
    for (int j = 0; j < width; j++) out[r * width + j] = j < (int)rk[r].size() ? rk[r][j] : 0;
  return (int)rk.size();
}
void oracle_p2_diag(int width, uint32_t* out) {
  auto d = p2_diag(width);
  for (int i = 0; i < width; i++) out[i] = d[i];
}
void oracle_keccak256(const uint8_t* msg, size_t len, uint8_t* out) { keccak256(msg, len, out); }
uint32_t oracle_root_of_unity(uint64_t n) { return root_of_unity(n); }

// Montgomery words in/out.
void oracle_rs_encode(const uint32_t* in, size_t n, size_t big, uint32_t* out) {
  std::vector<uint32_t> v(n);
  for (size_t i = 0; i < n; i++) v[i] = from_mont(in[i]);
  auto r = rs_encode(v.data(), n, big);
  for (size_t i = 0; i < big; i++) out[i] = to_mont(r[i]);
}
void oracle_rs_encode_e6(const uint32_t* in, size_t n, size_t big, uint32_t* out) {
  std::vector<E6> v(n);
  for (size_t i = 0; i < n; i++) for (int k = 0; k < 6; k++) v[i].c[k] = from_mont(in[6 * i + k]);
  auto r = rs_encode_e6(v.data(), n, big);
  for (size_t i = 0; i < big; i++) for (int k = 0; k < 6; k++) out[6 * i + k] = to_mont(r[i].c[k]);
}
void oracle_e6_mul(const uint32_t* a, const uint32_t* b, uint32_t* out) {
  E6 x, y;
  for (int k = 0; k < 6; k++) { x.c[k] = from_mont(a[k]); y.c[k] = from_mont(b[k]); }
  E6 z = e6_mul(x, y);
  for (int k = 0; k < 6; k++) out[k] = to_mont(z.c[k]);
}
void oracle_e6_inv(const uint32_t* a, uint32_t* out) {
  E6 x;
  for (int k = 0; k < 6; k++) x.c[k] = from_mont(a[k]);
  E6 z = e6_inv(x);
  for (int k = 0; k < 6; k++) out[k] = to_mont(z.c[k]);
}
// Sponge hash of `n` elements (Montgomery in, Montgomery digest out).
void oracle_sponge(const uint32_t* in, size_t n, uint32_t* out) {
  Sponge h;
  for (size_t i = 0; i < n; i++) h.write(from_mont(in[i]));
  Digest d = h.sum();
  for (int i = 0; i < 8; i++) out[i] = to_mont(d.v[i]);
}

// PCS.Commit of one batch (internal/fri/pcs.go:145-168).  groups[g] has
// rows[g] Lagrange-normal rows, nb[g] base and ne[g] ext columns; `cols`
// lists every column pointer group by group (base then ext).  Writes the
// root; when `leaves_out` is non-null, also the leaf digests of each group
// in sorted (size-descending, stable) order, concatenated.
int oracle_commit(uint32_t n_groups, const uint64_t* rows, const uint32_t* nb, const uint32_t* ne,
                  const uint32_t* const* cols, uint32_t* root_out, uint32_t* leaves_out) {
  try {
    size_t ci = 0;
    struct G { size_t n; std::vector<std::vector<uint32_t>> b; std::vector<std::vector<E6>> e; };
    std::vector<G> gs(n_groups);
    for (uint32_t g = 0; g < n_groups; g++) {
      gs[g].n = rows[g];
      for (uint32_t i = 0; i < nb[g]; i++) {
        const uint32_t* src = cols[ci++];
        std::vector<uint32_t> v(rows[g]);
        for (size_t r = 0; r < rows[g]; r++) v[r] = from_mont(src[r]);
        gs[g].b.push_back(v);
      }
      for (uint32_t i = 0; i < ne[g]; i++) {
        const uint32_t* src = cols[ci++];
        std::vector<E6> v(rows[g]);
        for (size_t r = 0; r < rows[g]; r++) for (int k = 0; k < 6; k++) v[r].c[k] = from_mont(src[6 * r + k]);
        gs[g].e.push_back(v);
      }
    }
    std::vector<size_t> order(n_groups);
    for (size_t i = 0; i < order.size(); i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return gs[a].n > gs[b].n; });
    std::vector<std::vector<Digest>> leaves;
    for (size_t gi : order) {
      size_t big = 4 * gs[gi].n;
      std::vector<std::vector<uint32_t>> lb;
      std::vector<std::vector<E6>> le;
      for (auto& v : gs[gi].b) lb.push_back(rs_encode(v.data(), gs[gi].n, big));
      for (auto& v : gs[gi].e) le.push_back(rs_encode_e6(v.data(), gs[gi].n, big));
      std::vector<Digest> lv(big / 2);
      for (size_t k = 0; k < big / 2; k++) {
        Sponge h;
        h.write((uint32_t)LEAF_TAG); h.write((uint32_t)(2 * lb.size())); h.write((uint32_t)(2 * le.size()));
        for (auto& c : lb) h.write(c[2 * k]);
        for (auto& c : lb) h.write(c[2 * k + 1]);
        for (auto& c : le) h.write_e6(c[2 * k]);
        for (auto& c : le) h.write_e6(c[2 * k + 1]);
        lv[k] = h.sum();
      }
      leaves.push_back(lv);
    }
    std::vector<Injection> inj;
    for (size_t k = 1; k < leaves.size(); k++) inj.push_back(Injection{leaves[k]});
    Tree t = build_tree(leaves[0], inj);
    for (int i = 0; i < 8; i++) root_out[i] = to_mont(t.root().v[i]);
    if (leaves_out) {
      size_t o = 0;
      for (auto& lv : leaves) for (auto& d : lv) for (int i = 0; i < 8; i++) leaves_out[o++] = to_mont(d.v[i]);
    }
    return 0;
  } catch (std::exception& e) {
    g_err = e.what();
    return 2;
  }
}

// Merkle root over `n` leaves (Montgomery digests) with injections of
// widths inj_w[k] whose leaves follow one another in `inj`.  Returns 0, or 2
// for a schedule merkle.NewWithInjections rejects (the reason in
// oracle_last_error()).
int oracle_merkle_root(const uint32_t* leaves, size_t n, uint32_t n_inj, const uint64_t* inj_w, const uint32_t* inj,
                       uint32_t* root_out) {
  try {
    auto rd = [](const uint32_t* p) { Digest d; for (int i = 0; i < 8; i++) d.v[i] = from_mont(p[i]); return d; };
    std::vector<Digest> lv(n);
    for (size_t i = 0; i < n; i++) lv[i] = rd(leaves + 8 * i);
    std::vector<Injection> ij;
    size_t o = 0;
    for (uint32_t k = 0; k < n_inj; k++) {
      Injection x;
      for (uint64_t i = 0; i < inj_w[k]; i++) { x.leaves.push_back(rd(inj + o)); o += 8; }
      ij.push_back(x);
    }
    Tree t = build_tree(lv, ij);
    for (int i = 0; i < 8; i++) root_out[i] = to_mont(t.root().v[i]);
    return 0;
  } catch (std::exception& e) {
    g_err = e.what();
    return 2;
  }
}

}  // extern "C"

extern "C" {
// One FRI fold of n E6 values in bit-reversed order, Montgomery in/out
// (internal/fri/fri.go:1177-1198).
void oracle_fri_fold(const uint32_t* layer, size_t n, const uint32_t* alpha, uint32_t* out) {
  E6 a;
  for (int k = 0; k < 6; k++) a.c[k] = from_mont(alpha[k]);
  size_t half = n / 2;
  int lg = 0;
  while ((1ull << lg) < half) lg++;
  uint32_t winv = inv(root_of_unity(n)), inv2 = inv(2);
  for (size_t i = 0; i < half; i++) {
    E6 p, q;
    for (int k = 0; k < 6; k++) { p.c[k] = from_mont(layer[6 * (2 * i) + k]); q.c[k] = from_mont(layer[6 * (2 * i + 1) + k]); }
    uint32_t xi = pow(winv, bitrev((uint32_t)i, lg));
    E6 s = e6_mul_base(e6_add(p, q), inv2);
    E6 d = e6_mul(e6_mul_base(e6_mul_base(e6_sub(p, q), inv2), xi), a);
    E6 r = e6_add(s, d);
    for (int k = 0; k < 6; k++) out[6 * i + k] = to_mont(r.c[k]);
  }
}
}

extern "C" {
// R[0] = 1, R[i] = prod_{k<i} num[k]/den[k] over E6 rows, Montgomery in/out
// (internal/poly/iop_utils.go:170-192,316-323).
void oracle_grand_product(const uint32_t* num, const uint32_t* den, size_t n, uint32_t* out) {
  E6 acc = e6_one();
  for (size_t i = 0; i < n; i++) {
    for (int k = 0; k < 6; k++) out[6 * i + k] = to_mont(acc.c[k]);
    E6 a, b;
    for (int k = 0; k < 6; k++) { a.c[k] = from_mont(num[6 * i + k]); b.c[k] = from_mont(den[6 * i + k]); }
    acc = e6_mul(acc, e6_mul(a, e6_inv(b)));
  }
}
}

extern "C" {
// Single-point DEEP quotient over base LDE columns of `rows` bit-reversed
// evaluations (internal/fri/deep.go:205-266), Montgomery in/out.
void oracle_deep_quotient(const uint32_t* lde, uint32_t n_cols, size_t rows, const uint32_t* alpha_m,
                          const uint32_t* z_m, const uint32_t* values_m, uint32_t* out) {
  E6 a, z;
  for (int k = 0; k < 6; k++) { a.c[k] = from_mont(alpha_m[k]); z.c[k] = from_mont(z_m[k]); }
  int lg = 0;
  while ((1ull << lg) < rows) lg++;
  uint32_t w = root_of_unity(rows);
  for (size_t r = 0; r < rows; r++) {
    uint32_t x = pow(w, bitrev((uint32_t)r, lg));
    E6 num = e6_zero(), run = e6_one();
    for (uint32_t i = 0; i < n_cols; i++) {
      E6 v;
      for (int k = 0; k < 6; k++) v.c[k] = from_mont(values_m[6 * i + k]);
      uint32_t p = from_mont(lde[(size_t)i * rows + r]);
      num = e6_add(num, e6_sub(e6_mul(run, v), e6_mul_base(run, p)));
      run = e6_mul(run, a);
    }
    E6 q = e6_mul(num, e6_inv(e6_sub(z, e6_from_base(x))));
    for (int k = 0; k < 6; k++) out[6 * r + k] = to_mont(q.c[k]);
  }
}
}
