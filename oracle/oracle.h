// CPU oracle for the loom Poseidon2 prove path — TEST INFRASTRUCTURE ONLY.
//
// This directory restates, in plain C++, the reference Go prover's algorithm
// for the Poseidon2 backend (github.com/consensys/loom) so that the CUDA
// implementation in loom_b200/ can be checked byte for byte.  Only tests/,
// __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it; the
// product library never links it.
//
// Arithmetic here is deliberately written differently from the product: the
// oracle keeps field elements as canonical integers in [0, p) and reduces
// with a 64-bit `%`, while the GPU keeps Montgomery words.  Conversions happen
// only at the boundary (inputs arrive as Montgomery words, the layout that
// gnark-crypto's koalabear.Element stores).
//
// Parity status (pins):
//  * Poseidon2 width-24 round keys: derived by the Keccak-256 chain of the
//    gnark-crypto parameter seed; the same derivation reproduces all 432
//    width-16 keys listed in the reference's
//    integration_test/zkc/riscv/zkc/lib/poseidon2/constants.zkc (tests pin it).
//  * Linear layers and diagonal: recursion/p2_air.go:80-117,
//    recursion/poseidon2.go:48-90 (width-16 diagonal pinned against the same
//    zkc file).
//  * E6 tower u^2 = 3, v^3 = u + 1: recursion/e6.go:21-53.
//  * 2-adic root of unity 3^127 and multiplicative generator 3: derived from
//    the field (3 is the smallest generator of F_p^*); no reference test
//    vector holds them ("parity unpinned" for these two constants).
#pragma once
#include <cstdint>
#include <cstddef>
#include <string>
#include <vector>

namespace orc {

static constexpr uint32_t P = 0x7f000001u;  // 2^31 - 2^24 + 1

inline uint32_t add(uint32_t a, uint32_t b) { uint32_t s = a + b; return s >= P ? s - P : s; }
inline uint32_t sub(uint32_t a, uint32_t b) { return a >= b ? a - b : a + P - b; }
inline uint32_t neg(uint32_t a) { return a ? P - a : 0; }
inline uint32_t mul(uint32_t a, uint32_t b) { return (uint32_t)(((uint64_t)a * b) % P); }
uint32_t pow(uint32_t a, uint64_t e);
uint32_t inv(uint32_t a);  // a^(p-2); inv(0) = 0

// Montgomery words (R = 2^32) <-> canonical values.
uint32_t to_mont(uint32_t a);
uint32_t from_mont(uint32_t m);

// E6 = E2[v]/(v^3 - (u+1)), E2 = F[u]/(u^2 - 3).
// Layout [B0.A0, B0.A1, B1.A0, B1.A1, B2.A0, B2.A1] (internal/hash/hash.go:59-68).
struct E6 { uint32_t c[6]; };
E6 e6_zero();
E6 e6_one();
E6 e6_from_base(uint32_t a);
E6 e6_add(const E6& a, const E6& b);
E6 e6_sub(const E6& a, const E6& b);
E6 e6_mul(const E6& a, const E6& b);
E6 e6_mul_base(const E6& a, uint32_t b);
E6 e6_inv(const E6& a);
E6 e6_pow(const E6& a, uint64_t e);
bool e6_eq(const E6& a, const E6& b);
bool e6_is_zero(const E6& a);

// Domains: generator of the subgroup of order n = 2^k (k <= 24).
uint32_t root_of_unity(uint64_t n);
static constexpr uint32_t MULT_GEN = 3;  // generator of F_p^*

// ---------------------------------------------------------------- Poseidon2
static constexpr int P2_W = 24, P2_RATE = 16, P2_FULL = 6, P2_PARTIAL = 21, DIGEST = 8;
struct Digest { uint32_t v[8]; };
bool digest_eq(const Digest& a, const Digest& b);

void keccak256(const uint8_t* msg, size_t len, uint8_t out[32]);
// Round keys of gnark-crypto's koalabear Poseidon2 for (width, rF, rP):
// rows of `width` keys for full rounds, rows of 1 key for partial rounds.
std::vector<std::vector<uint32_t>> p2_round_keys(int width, int rf, int rp);
std::vector<uint32_t> p2_diag(int width);  // internal-matrix diagonal, canonical
void p2_permute(uint32_t* state, int width);  // width 16 or 24, canonical values

// Width-24, rate-16 overwrite-mode sponge without padding
// (internal/hash/poseidon2.go:165-255).
struct Sponge {
  uint32_t state[24];
  uint32_t block[16];
  int block_len = 0;
  bool wrote = false;
  Sponge() { reset(); }
  void reset();
  void write(uint32_t x);
  void write_e6(const E6& x) { for (int i = 0; i < 6; i++) write(x.c[i]); }
  Digest sum();
};
Digest node_compress(uint64_t tag, const Digest& l, const Digest& r);
static constexpr uint64_t LEAF_TAG = 0x4c454146, NODE_TAG = 0x4e4f4445;

// ---------------------------------------------------------------- NTT
uint32_t bitrev(uint32_t x, int logn);
void bit_reverse(uint32_t* a, size_t n);
void bit_reverse_e6(E6* a, size_t n);
// gnark-crypto conventions: FFT DIF natural -> bit-reversed; inverse DIF
// natural -> bit-reversed scaled by 1/n; FFT DIT bit-reversed -> natural.
void fft_dif(uint32_t* a, size_t n);
void ifft_dif(uint32_t* a, size_t n);
void fft_dit(uint32_t* a, size_t n);
void fft_dif_e6(E6* a, size_t n);
void ifft_dif_e6(E6* a, size_t n);
// Reed-Solomon encode (internal/reedsolomon/rs.go:52-87).
std::vector<uint32_t> rs_encode(const uint32_t* p, size_t n, size_t big);
std::vector<E6> rs_encode_e6(const E6* p, size_t n, size_t big);

// ---------------------------------------------------------------- Merkle
struct Injection { std::vector<Digest> leaves; };
struct Tree {
  size_t n_leaves = 0;
  std::vector<Digest> nodes;           // 1-indexed, size 2*n_leaves
  std::vector<Injection> injections;   // non-increasing widths
  Digest root() const { return nodes[1]; }
};
Tree build_tree(const std::vector<Digest>& leaves, const std::vector<Injection>& inj);
struct MerklePath {
  uint32_t leaf_idx;
  std::vector<Digest> siblings;
  std::vector<Digest> injection_leaves;
};
MerklePath open_path(const Tree& t, size_t idx);

// ---------------------------------------------------------------- transcript
std::vector<uint32_t> string_to_elements(uint64_t tag, const std::string& s);
struct Transcript {
  struct Ch { std::string name; std::vector<uint32_t> bindings; Digest value; bool done = false; };
  std::vector<Ch> chs;
  int find(const std::string& n) const;
  void new_challenge(const std::string& n);
  void bind(const std::string& n, const uint32_t* v, size_t len);
  void bind(const std::string& n, const std::vector<uint32_t>& v) { bind(n, v.data(), v.size()); }
  Digest compute(const std::string& n);
};
E6 digest_to_e6(const Digest& d);

}  // namespace orc
