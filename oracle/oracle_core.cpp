// CPU oracle (test infrastructure): field, E6, Keccak, Poseidon2, sponge,
// NTT, Merkle tree and Fiat-Shamir transcript.  See oracle.h for the role of
// this code and its pins.  Reference files cited per function are paths
// inside github.com/consensys/loom.
#include "oracle.h"

#include <cstring>
#include <stdexcept>

namespace orc {

uint32_t pow(uint32_t a, uint64_t e) {
  uint32_t r = 1, b = a;
  while (e) { if (e & 1) r = mul(r, b); b = mul(b, b); e >>= 1; }
  return r;
}
uint32_t inv(uint32_t a) { return a ? pow(a, P - 2) : 0; }

uint32_t to_mont(uint32_t a) { return (uint32_t)(((uint64_t)a << 32) % P); }
uint32_t from_mont(uint32_t m) {
  static const uint32_t rinv = inv(to_mont(1));  // (2^32)^-1 mod p
  return mul(m % P, rinv);
}

// ---------------------------------------------------------------- E2 / E6
// E2 element (a0 + a1*u), u^2 = 3.
struct E2 { uint32_t a0, a1; };
static inline E2 e2_add(E2 x, E2 y) { return {add(x.a0, y.a0), add(x.a1, y.a1)}; }
static inline E2 e2_sub(E2 x, E2 y) { return {sub(x.a0, y.a0), sub(x.a1, y.a1)}; }
static inline E2 e2_mul(E2 x, E2 y) {
  return {add(mul(x.a0, y.a0), mul(3, mul(x.a1, y.a1))), add(mul(x.a0, y.a1), mul(x.a1, y.a0))};
}
// xi = 1 + u: (p + q u)(1 + u) = (p + 3q) + (p + q) u  (recursion/e6.go:30-33)
static inline E2 e2_mul_xi(E2 x) { return {add(x.a0, mul(3, x.a1)), add(x.a0, x.a1)}; }
static inline E2 e2_inv(E2 x) {
  uint32_t n = sub(mul(x.a0, x.a0), mul(3, mul(x.a1, x.a1)));
  uint32_t ni = inv(n);
  return {mul(x.a0, ni), mul(neg(x.a1), ni)};
}
static inline E2 g2(const E6& a, int i) { return {a.c[2 * i], a.c[2 * i + 1]}; }
static inline void s2(E6& a, int i, E2 v) { a.c[2 * i] = v.a0; a.c[2 * i + 1] = v.a1; }

E6 e6_zero() { E6 r; memset(r.c, 0, sizeof r.c); return r; }
E6 e6_one() { E6 r = e6_zero(); r.c[0] = 1; return r; }
E6 e6_from_base(uint32_t a) { E6 r = e6_zero(); r.c[0] = a; return r; }
E6 e6_add(const E6& a, const E6& b) { E6 r; for (int i = 0; i < 6; i++) r.c[i] = add(a.c[i], b.c[i]); return r; }
E6 e6_sub(const E6& a, const E6& b) { E6 r; for (int i = 0; i < 6; i++) r.c[i] = sub(a.c[i], b.c[i]); return r; }
E6 e6_mul_base(const E6& a, uint32_t b) { E6 r; for (int i = 0; i < 6; i++) r.c[i] = mul(a.c[i], b); return r; }
bool e6_eq(const E6& a, const E6& b) { return memcmp(a.c, b.c, sizeof a.c) == 0; }
bool e6_is_zero(const E6& a) { for (int i = 0; i < 6; i++) if (a.c[i]) return false; return true; }

// Schoolbook product over E2 with v^3 = xi (recursion/e6.go:24-53).
E6 e6_mul(const E6& x, const E6& y) {
  E2 p[3][3];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) p[i][j] = e2_mul(g2(x, i), g2(y, j));
  E6 r;
  s2(r, 0, e2_add(p[0][0], e2_mul_xi(e2_add(p[1][2], p[2][1]))));
  s2(r, 1, e2_add(e2_add(p[0][1], p[1][0]), e2_mul_xi(p[2][2])));
  s2(r, 2, e2_add(e2_add(p[0][2], p[1][1]), p[2][0]));
  return r;
}

// Inverse in the cubic extension: (c0, c1, c2) / (a0 c0 + xi (a2 c1 + a1 c2)).
E6 e6_inv(const E6& a) {
  E2 a0 = g2(a, 0), a1 = g2(a, 1), a2 = g2(a, 2);
  E2 c0 = e2_sub(e2_mul(a0, a0), e2_mul_xi(e2_mul(a1, a2)));
  E2 c1 = e2_sub(e2_mul_xi(e2_mul(a2, a2)), e2_mul(a0, a1));
  E2 c2 = e2_sub(e2_mul(a1, a1), e2_mul(a0, a2));
  E2 t = e2_add(e2_mul(a0, c0), e2_mul_xi(e2_add(e2_mul(a2, c1), e2_mul(a1, c2))));
  E2 ti = e2_inv(t);
  E6 r;
  s2(r, 0, e2_mul(c0, ti));
  s2(r, 1, e2_mul(c1, ti));
  s2(r, 2, e2_mul(c2, ti));
  return r;
}
E6 e6_pow(const E6& a, uint64_t e) {
  E6 r = e6_one(), b = a;
  while (e) { if (e & 1) r = e6_mul(r, b); b = e6_mul(b, b); e >>= 1; }
  return r;
}

uint32_t root_of_unity(uint64_t n) {
  // 3^((p-1)/2^24) generates the subgroup of order 2^24; smaller subgroups
  // take the matching power.
  int logn = 0;
  while ((1ull << logn) < n) logn++;
  if (logn > 24) throw std::runtime_error("root_of_unity: order above 2^24");
  uint32_t w = pow(MULT_GEN, (P - 1) >> 24);
  for (int i = logn; i < 24; i++) w = mul(w, w);
  return w;
}

// ---------------------------------------------------------------- Keccak-256
// Original Keccak (0x01 domain padding), as used by gnark-crypto to derive
// Poseidon2 round keys.  Written from the Keccak reference specification.
static const uint64_t KRC[24] = {
    0x0000000000000001ull, 0x0000000000008082ull, 0x800000000000808Aull, 0x8000000080008000ull,
    0x000000000000808Bull, 0x0000000080000001ull, 0x8000000080008081ull, 0x8000000000008009ull,
    0x000000000000008Aull, 0x0000000000000088ull, 0x0000000080008009ull, 0x000000008000000Aull,
    0x000000008000808Bull, 0x800000000000008Bull, 0x8000000000008089ull, 0x8000000000008003ull,
    0x8000000000008002ull, 0x8000000000000080ull, 0x000000000000800Aull, 0x800000008000000Aull,
    0x8000000080008081ull, 0x8000000000008080ull, 0x0000000080000001ull, 0x8000000080008008ull};
static const int KROT[5][5] = {{0, 36, 3, 41, 18}, {1, 44, 10, 45, 2}, {62, 6, 43, 15, 61},
                               {28, 55, 25, 21, 56}, {27, 20, 39, 8, 14}};
static inline uint64_t rol(uint64_t x, int n) { return n ? (x << n) | (x >> (64 - n)) : x; }
static void keccak_f(uint64_t A[5][5]) {
  for (int rnd = 0; rnd < 24; rnd++) {
    uint64_t C[5], D[5], B[5][5];
    for (int x = 0; x < 5; x++) C[x] = A[x][0] ^ A[x][1] ^ A[x][2] ^ A[x][3] ^ A[x][4];
    for (int x = 0; x < 5; x++) D[x] = C[(x + 4) % 5] ^ rol(C[(x + 1) % 5], 1);
    for (int x = 0; x < 5; x++)
      for (int y = 0; y < 5; y++) A[x][y] ^= D[x];
    for (int x = 0; x < 5; x++)
      for (int y = 0; y < 5; y++) B[y][(2 * x + 3 * y) % 5] = rol(A[x][y], KROT[x][y]);
    for (int x = 0; x < 5; x++)
      for (int y = 0; y < 5; y++) A[x][y] = B[x][y] ^ ((~B[(x + 1) % 5][y]) & B[(x + 2) % 5][y]);
    A[0][0] ^= KRC[rnd];
  }
}
void keccak256(const uint8_t* msg, size_t len, uint8_t out[32]) {
  const size_t rate = 136;
  std::vector<uint8_t> m(msg, msg + len);
  m.push_back(0x01);
  while (m.size() % rate) m.push_back(0);
  m.back() |= 0x80;
  uint64_t A[5][5];
  memset(A, 0, sizeof A);
  for (size_t off = 0; off < m.size(); off += rate) {
    for (size_t i = 0; i < rate / 8; i++) {
      uint64_t w = 0;
      for (int b = 0; b < 8; b++) w |= (uint64_t)m[off + 8 * i + b] << (8 * b);
      A[i % 5][i / 5] ^= w;
    }
    keccak_f(A);
  }
  for (int i = 0; i < 4; i++)
    for (int b = 0; b < 8; b++) out[8 * i + b] = (uint8_t)(A[i % 5][i / 5] >> (8 * b));
}

// ---------------------------------------------------------------- Poseidon2
// Round keys: seed "Poseidon2-koalabear[t=W,rF=F,rP=R,d=3]", h0 = keccak(seed),
// key_i = big-endian(h_i) mod p with h_i = keccak(h_{i-1}); full rounds take W
// keys, partial rounds one key (call sites internal/hash/poseidon2.go:51-54).
std::vector<std::vector<uint32_t>> p2_round_keys(int width, int rf, int rp) {
  std::string seed = "Poseidon2-koalabear[t=" + std::to_string(width) + ",rF=" + std::to_string(rf) +
                     ",rP=" + std::to_string(rp) + ",d=3]";
  uint8_t h[32];
  keccak256((const uint8_t*)seed.data(), seed.size(), h);
  auto next = [&]() {
    uint8_t t[32];
    keccak256(h, 32, t);
    memcpy(h, t, 32);
    uint32_t r = 0;
    for (int i = 0; i < 32; i++) r = (uint32_t)((((uint64_t)r << 8) | h[i]) % P);
    return r;
  };
  std::vector<std::vector<uint32_t>> rk;
  for (int r = 0; r < rf / 2; r++) { std::vector<uint32_t> row; for (int j = 0; j < width; j++) row.push_back(next()); rk.push_back(row); }
  for (int r = 0; r < rp; r++) rk.push_back({next()});
  for (int r = 0; r < rf / 2; r++) { std::vector<uint32_t> row; for (int j = 0; j < width; j++) row.push_back(next()); rk.push_back(row); }
  return rk;
}

// Internal diagonal M_I = 1.1^T + diag (recursion/poseidon2.go:48-90).
std::vector<uint32_t> p2_diag(int w) {
  std::vector<int> pos, negs;
  if (w == 16) { pos = {8, 3, 24}; negs = {8, 3, 4, 24}; }
  else if (w == 24) { pos = {8, 2, 3, 4, 5, 6, 24}; negs = {8, 3, 4, 5, 6, 7, 9, 24}; }
  else throw std::runtime_error("p2_diag: width");
  std::vector<uint32_t> d(w);
  auto ip2 = [](int n) { return inv(pow(2, n)); };
  d[0] = neg(2); d[1] = 1; d[2] = 2; d[3] = ip2(1); d[4] = 3; d[5] = 4;
  d[6] = neg(ip2(1)); d[7] = neg(3); d[8] = neg(4);
  for (size_t i = 0; i < pos.size(); i++) d[9 + i] = ip2(pos[i]);
  for (size_t i = 0; i < negs.size(); i++) d[9 + pos.size() + i] = neg(ip2(negs[i]));
  return d;
}

// circ(2 M4, M4, ...) with M4 = [[2,3,1,1],[1,2,3,1],[1,1,2,3],[3,1,1,2]]
// (recursion/p2_air.go:80-104), written as the dense 4x4 product.
static void mat_external(uint32_t* s, int w) {
  static const uint32_t M4[4][4] = {{2, 3, 1, 1}, {1, 2, 3, 1}, {1, 1, 2, 3}, {3, 1, 1, 2}};
  for (int c = 0; c < w / 4; c++) {
    uint32_t x[4], y[4];
    for (int i = 0; i < 4; i++) x[i] = s[4 * c + i];
    for (int r = 0; r < 4; r++) {
      uint32_t acc = 0;
      for (int j = 0; j < 4; j++) acc = add(acc, mul(M4[r][j], x[j]));
      y[r] = acc;
    }
    for (int i = 0; i < 4; i++) s[4 * c + i] = y[i];
  }
  uint32_t sums[4] = {0, 0, 0, 0};
  for (int c = 0; c < w / 4; c++)
    for (int j = 0; j < 4; j++) sums[j] = add(sums[j], s[4 * c + j]);
  for (int i = 0; i < w; i++) s[i] = add(s[i], sums[i % 4]);
}
static void mat_internal(uint32_t* s, int w, const std::vector<uint32_t>& d) {
  uint32_t sum = 0;
  for (int i = 0; i < w; i++) sum = add(sum, s[i]);
  for (int i = 0; i < w; i++) s[i] = add(sum, mul(s[i], d[i]));
}
static inline uint32_t cube(uint32_t x) { return mul(mul(x, x), x); }

// M_E; 3 full rounds; 21 partial rounds (lane 0); 3 full rounds; S-box x^3
// (recursion/p2_air.go:206-300).
void p2_permute(uint32_t* s, int w) {
  static const auto rk16 = p2_round_keys(16, 6, 21), rk24 = p2_round_keys(24, 6, 21);
  static const auto d16 = p2_diag(16), d24 = p2_diag(24);
  const auto& rk = w == 16 ? rk16 : rk24;
  const auto& d = w == 16 ? d16 : d24;
  mat_external(s, w);
  for (int r = 0; r < 27; r++) {
    bool full = r < 3 || r >= 24;
    if (full) {
      for (int i = 0; i < w; i++) s[i] = cube(add(s[i], rk[r][i]));
      mat_external(s, w);
    } else {
      s[0] = cube(add(s[0], rk[r][0]));
      mat_internal(s, w, d);
    }
  }
}

bool digest_eq(const Digest& a, const Digest& b) { return memcmp(a.v, b.v, sizeof a.v) == 0; }

void Sponge::reset() {
  memset(state, 0, sizeof state);
  memset(block, 0, sizeof block);
  block_len = 0;
  wrote = false;
}
void Sponge::write(uint32_t x) {
  block[block_len++] = x;
  if (block_len == P2_RATE) {
    memcpy(state, block, sizeof block);
    p2_permute(state, 24);
    memset(block, 0, sizeof block);
    block_len = 0;
    wrote = true;
  }
}
Digest Sponge::sum() {
  Digest d;
  if (!wrote && block_len == 0) { memset(d.v, 0, sizeof d.v); return d; }
  if (block_len > 0) {
    for (int i = 0; i < block_len; i++) state[i] = block[i];
    p2_permute(state, 24);
    memset(block, 0, sizeof block);
    block_len = 0;
    wrote = true;
  }
  memcpy(d.v, state, sizeof d.v);
  return d;
}

// state = [tag, 0 x7, left, right]; digest = first 8 lanes after one
// permutation (internal/hash/poseidon2.go:409-422).
Digest node_compress(uint64_t tag, const Digest& l, const Digest& r) {
  uint32_t s[24];
  memset(s, 0, sizeof s);
  s[0] = (uint32_t)(tag % P);
  for (int i = 0; i < 8; i++) { s[8 + i] = l.v[i]; s[16 + i] = r.v[i]; }
  p2_permute(s, 24);
  Digest d;
  memcpy(d.v, s, sizeof d.v);
  return d;
}

// ---------------------------------------------------------------- NTT
uint32_t bitrev(uint32_t x, int logn) {
  uint32_t r = 0;
  for (int i = 0; i < logn; i++) { r = (r << 1) | (x & 1); x >>= 1; }
  return r;
}
static int ilog2(size_t n) { int k = 0; while ((1ull << k) < n) k++; return k; }
template <class T> static void bitrev_t(T* a, size_t n) {
  int lg = ilog2(n);
  for (size_t i = 0; i < n; i++) { size_t j = bitrev((uint32_t)i, lg); if (i < j) std::swap(a[i], a[j]); }
}
void bit_reverse(uint32_t* a, size_t n) { bitrev_t(a, n); }
void bit_reverse_e6(E6* a, size_t n) { bitrev_t(a, n); }

static inline uint32_t mb(uint32_t a, uint32_t b) { return mul(a, b); }
static inline E6 mb(const E6& a, uint32_t b) { return e6_mul_base(a, b); }
static inline uint32_t ad(uint32_t a, uint32_t b) { return add(a, b); }
static inline E6 ad(const E6& a, const E6& b) { return e6_add(a, b); }
static inline uint32_t sb(uint32_t a, uint32_t b) { return sub(a, b); }
static inline E6 sb(const E6& a, const E6& b) { return e6_sub(a, b); }

// Gentleman-Sande: natural input, bit-reversed output, X_k = sum a_j w^(jk).
template <class T> static void dif_t(T* a, size_t n, uint32_t w) {
  for (size_t len = n; len >= 2; len >>= 1) {
    uint32_t wl = pow(w, n / len);
    for (size_t i = 0; i < n; i += len) {
      uint32_t t = 1;
      for (size_t j = 0; j < len / 2; j++) {
        T u = a[i + j], v = a[i + j + len / 2];
        a[i + j] = ad(u, v);
        a[i + j + len / 2] = mb(sb(u, v), t);
        t = mul(t, wl);
      }
    }
  }
}
// Cooley-Tukey: bit-reversed input, natural output.
template <class T> static void dit_t(T* a, size_t n, uint32_t w) {
  for (size_t len = 2; len <= n; len <<= 1) {
    uint32_t wl = pow(w, n / len);
    for (size_t i = 0; i < n; i += len) {
      uint32_t t = 1;
      for (size_t j = 0; j < len / 2; j++) {
        T u = a[i + j], v = mb(a[i + j + len / 2], t);
        a[i + j] = ad(u, v);
        a[i + j + len / 2] = sb(u, v);
        t = mul(t, wl);
      }
    }
  }
}
void fft_dif(uint32_t* a, size_t n) { dif_t(a, n, root_of_unity(n)); }
void fft_dit(uint32_t* a, size_t n) { dit_t(a, n, root_of_unity(n)); }
void ifft_dif(uint32_t* a, size_t n) {
  dif_t(a, n, inv(root_of_unity(n)));
  uint32_t ni = inv((uint32_t)(n % P));
  for (size_t i = 0; i < n; i++) a[i] = mul(a[i], ni);
}
void fft_dif_e6(E6* a, size_t n) { dif_t(a, n, root_of_unity(n)); }
void ifft_dif_e6(E6* a, size_t n) {
  dif_t(a, n, inv(root_of_unity(n)));
  uint32_t ni = inv((uint32_t)(n % P));
  for (size_t i = 0; i < n; i++) a[i] = e6_mul_base(a[i], ni);
}

// iFFT_DIF(n) -> BitReverse -> zero-pad -> FFT_DIF(big): bit-reversed
// evaluations on the subgroup of order `big` (internal/reedsolomon/rs.go:52-70).
std::vector<uint32_t> rs_encode(const uint32_t* p, size_t n, size_t big) {
  std::vector<uint32_t> r(big, 0);
  for (size_t i = 0; i < n; i++) r[i] = p[i];
  ifft_dif(r.data(), n);
  bit_reverse(r.data(), n);
  fft_dif(r.data(), big);
  return r;
}
std::vector<E6> rs_encode_e6(const E6* p, size_t n, size_t big) {
  std::vector<E6> r(big, e6_zero());
  for (size_t i = 0; i < n; i++) r[i] = p[i];
  ifft_dif_e6(r.data(), n);
  bit_reverse_e6(r.data(), n);
  fft_dif_e6(r.data(), big);
  return r;
}

// ---------------------------------------------------------------- Merkle
// Flat 1-indexed tree; after the leaves and after every 2-to-1 level, the
// injections of that width fold in schedule order: node = H(node, inj)
// (internal/merkle/tree.go:210-327).
Tree build_tree(const std::vector<Digest>& leaves, const std::vector<Injection>& inj) {
  Tree t;
  size_t n = leaves.size();
  if (n == 0 || (n & (n - 1))) throw std::runtime_error("build_tree: leaves must be a power of two");
  size_t prev = n;
  for (auto& j : inj) {
    size_t w = j.leaves.size();
    if (w == 0 || (w & (w - 1)) || w > prev) throw std::runtime_error("build_tree: bad injection widths");
    prev = w;
  }
  t.n_leaves = n;
  t.injections = inj;
  t.nodes.assign(2 * n, Digest{});
  for (size_t i = 0; i < n; i++) t.nodes[n + i] = leaves[i];
  size_t next = 0;
  // Nodes of one level are independent, and so are the injection chains of
  // one width (each node folds its own chain in schedule order): both run
  // over the host threads.
  auto fold = [&](size_t start) {
    size_t first = next;
    while (next < inj.size() && inj[next].leaves.size() == start) next++;
    if (next == first) return;
#pragma omp parallel for schedule(static) if (start >= 256)
    for (size_t j = 0; j < start; j++)
      for (size_t k = first; k < next; k++)
        t.nodes[start + j] = node_compress(NODE_TAG, t.nodes[start + j], inj[k].leaves[j]);
  };
  fold(n);
  for (size_t start = n >> 1; start >= 1; start >>= 1) {
#pragma omp parallel for schedule(static) if (start >= 256)
    for (size_t i = start; i < 2 * start; i++) t.nodes[i] = node_compress(NODE_TAG, t.nodes[2 * i], t.nodes[2 * i + 1]);
    fold(start);
  }
  return t;
}
// internal/merkle/tree.go:341-368
MerklePath open_path(const Tree& t, size_t idx) {
  MerklePath p;
  p.leaf_idx = (uint32_t)idx;
  size_t pos = t.n_leaves + idx;
  int depth = ilog2(t.n_leaves);
  for (int k = 0; k < depth; k++) { p.siblings.push_back(t.nodes[pos ^ 1]); pos >>= 1; }
  for (auto& inj : t.injections) {
    int d = ilog2(t.n_leaves / inj.leaves.size());
    p.injection_leaves.push_back(inj.leaves[idx >> d]);
  }
  return p;
}

// ---------------------------------------------------------------- transcript
// internal/hash/hash.go:39-58
std::vector<uint32_t> string_to_elements(uint64_t tag, const std::string& s) {
  std::vector<uint32_t> r;
  r.push_back((uint32_t)(tag % P));
  r.push_back((uint32_t)(s.size() % P));
  for (size_t i = 0; i < s.size(); i += 3) {
    uint64_t limb = 0;
    for (size_t j = 0; j < 3 && i + j < s.size(); j++) limb |= (uint64_t)(uint8_t)s[i + j] << (8 * j);
    r.push_back((uint32_t)(limb % P));
  }
  return r;
}
int Transcript::find(const std::string& n) const {
  for (size_t i = 0; i < chs.size(); i++) if (chs[i].name == n) return (int)i;
  return -1;
}
void Transcript::new_challenge(const std::string& n) {
  if (find(n) >= 0) throw std::runtime_error("transcript: duplicate challenge " + n);
  Ch c; c.name = n; chs.push_back(c);
}
void Transcript::bind(const std::string& n, const uint32_t* v, size_t len) {
  int i = find(n);
  if (i < 0) throw std::runtime_error("transcript: unknown challenge " + n);
  if (chs[i].done) throw std::runtime_error("transcript: challenge already computed " + n);
  chs[i].bindings.insert(chs[i].bindings.end(), v, v + len);
}
// H(FSID-tagged name || previous challenge || bindings)
// (internal/fiat-shamir/transcript.go:285-315)
Digest Transcript::compute(const std::string& n) {
  int i = find(n);
  if (i < 0) throw std::runtime_error("transcript: unknown challenge " + n);
  if (chs[i].done) return chs[i].value;
  Sponge h;
  for (uint32_t x : string_to_elements(0x46534944, n)) h.write(x);
  if (i != 0) {
    if (!chs[i - 1].done) throw std::runtime_error("transcript: previous challenge not computed for " + n);
    for (int k = 0; k < 8; k++) h.write(chs[i - 1].value.v[k]);
  }
  for (uint32_t x : chs[i].bindings) h.write(x);
  chs[i].value = h.sum();
  chs[i].done = true;
  return chs[i].value;
}
E6 digest_to_e6(const Digest& d) { E6 r; for (int i = 0; i < 6; i++) r.c[i] = d.v[i]; return r; }

}  // namespace orc
